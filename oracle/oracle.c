/*
 * CPU oracle for the Renderer2 filter path — TEST INFRASTRUCTURE ONLY (see
 * oracle.h).  Plain C11; compiled with -ffp-contract=off so every float
 * expression rounds like the device code (which is built with -fmad=false).
 */
#include "oracle.h"
#include "oracle_internal.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* ---------------------------------------------------------------- Philox */

void orc_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

#define u01 oi_u01

/* sin/cos of u turns: Taylor series on [-pi/4, pi/4] after exact quadrant
 * reduction; the same operation sequence as the device code. */
void orc_sincos_turns(float u, float* s, float* c) {
  float q = rintf(u * 4.0f);
  float r = u - q * 0.25f;
  float t = r * 6.28318548f;
  float t2 = t * t;
  float ps = fmaf(t2, 2.75573192e-6f, -1.98412698e-4f);
  ps = fmaf(t2, ps, 8.33333333e-3f);
  ps = fmaf(t2, ps, -1.66666667e-1f);
  float sn = fmaf(t * t2, ps, t);
  float pc = fmaf(t2, -2.75573192e-7f, 2.48015873e-5f);
  pc = fmaf(t2, pc, -1.38888889e-3f);
  pc = fmaf(t2, pc, 4.16666667e-2f);
  pc = fmaf(t2, pc, -0.5f);
  float cs = fmaf(t2, pc, 1.0f);
  int qi = ((int)q) & 3;
  if (qi == 0) { *s = sn; *c = cs; }
  else if (qi == 1) { *s = cs; *c = -sn; }
  else if (qi == 2) { *s = -sn; *c = -cs; }
  else { *s = -cs; *c = sn; }
}

/* ---------------------------------------------------------------- vectors */

/* ---------------------------------------------------------------- LBVH */

#define SAH_NODE 1.2f
#define SAH_TRI 1.0f
#define LEAF_MAX 8
#define BVH_NONE ((int32_t)0x80000000)
#define BVH_STACK 96

typedef struct { uint64_t key; uint32_t idx; } kv_t;
static int kv_cmp(const void* a, const void* b) {
  const kv_t* x = (const kv_t*)a;
  const kv_t* y = (const kv_t*)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->idx < y->idx ? -1 : (x->idx > y->idx ? 1 : 0);
}

static uint64_t expand21(uint32_t v) {
  uint64_t x = v & 0x1FFFFFu;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

static uint32_t quant21(float c, float cmin, float inv) {
  float q = (c - cmin) * inv * 2097152.0f;
  q = fminf(fmaxf(q, 0.0f), 2097151.0f);
  return (uint32_t)q;
}

static int kdelta(const uint64_t* k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  if (k[i] == k[j]) return 64 + __builtin_clz((uint32_t)(i ^ j));
  return __builtin_clzll(k[i] ^ k[j]);
}

typedef struct {
  int n;
  int *left, *right, *first, *last, *parent, *collapse, *height;
  float *lo, *hi, *cost;      /* internal nodes: 4 floats per box (x,y,z,0) */
  float *leafLo, *leafHi;     /* sorted leaves */
} bld_t;

static float box_area(const float* l, const float* h) {
  float dx = h[0] - l[0], dy = h[1] - l[1], dz = h[2] - l[2];
  return dx * dy + dy * dz + dz * dx;
}

static void child_info(const bld_t* B, int c, const float** lo, const float** hi, float* cost, int* height) {
  if (c < 0) {
    *lo = &B->leafLo[4 * (~c)];
    *hi = &B->leafHi[4 * (~c)];
    *cost = SAH_TRI;
    *height = 0;
  } else {
    *lo = &B->lo[4 * c];
    *hi = &B->hi[4 * c];
    *cost = B->cost[c];
    *height = B->height[c];
  }
}

static void bottom_up(bld_t* B, int p) {
  /* post-order via explicit stack to avoid deep recursion */
  int* st = (int*)malloc(sizeof(int) * 2 * (size_t)(B->n + 1));
  int sp = 0;
  st[sp++] = p;
  st[sp++] = 0;
  while (sp > 0) {
    int state = st[--sp];
    int node = st[--sp];
    if (state == 0) {
      st[sp++] = node;
      st[sp++] = 1;
      if (B->right[node] >= 0) { st[sp++] = B->right[node]; st[sp++] = 0; }
      if (B->left[node] >= 0) { st[sp++] = B->left[node]; st[sp++] = 0; }
    } else {
      const float *al, *ah, *bl, *bh;
      float ac, bc;
      int aht, bht;
      child_info(B, B->left[node], &al, &ah, &ac, &aht);
      child_info(B, B->right[node], &bl, &bh, &bc, &bht);
      float* lo = &B->lo[4 * node];
      float* hi = &B->hi[4 * node];
      for (int k = 0; k < 3; ++k) {
        lo[k] = fminf(al[k], bl[k]);
        hi[k] = fmaxf(ah[k], bh[k]);
      }
      lo[3] = hi[3] = 0.0f;
      float A = box_area(lo, hi);
      float Al = box_area(al, ah), Ar = box_area(bl, bh);
      float inner = (A > 0.0f) ? SAH_NODE + (Al * ac + Ar * bc) / A : SAH_NODE + ac + bc;
      int count = B->last[node] - B->first[node] + 1;
      float leafc = SAH_TRI * (float)count;
      int col = (count <= LEAF_MAX && leafc <= inner) ? 1 : 0;
      B->cost[node] = col ? leafc : inner;
      B->height[node] = col ? 0 : 1 + (aht > bht ? aht : bht);
      B->collapse[node] = col;
    }
  }
  free(st);
}

static int leaf_ref(int first, int count) { return ~(first | (count << 26)); }

static int child_ref(const bld_t* B, int c) {
  if (c < 0) return leaf_ref(~c, 1);
  if (B->collapse[c]) return leaf_ref(B->first[c], B->last[c] - B->first[c] + 1);
  return c;
}

static void put_box(int32_t* w, int slot, const float* l, const float* h) {
  /* slot 0: words 0..3 (lx hx ly hy) and 8,9 (lz hz); slot 1: words 4..7 and 10,11 */
  float* f = (float*)w;
  if (slot == 0) {
    f[0] = l[0]; f[1] = h[0]; f[2] = l[1]; f[3] = h[1]; f[8] = l[2]; f[9] = h[2];
  } else {
    f[4] = l[0]; f[5] = h[0]; f[6] = l[1]; f[7] = h[1]; f[10] = l[2]; f[11] = h[2];
  }
}

/* ------------------------------------------------ PLOC (bvh_ploc.cu) */
#define PLOC_RADIUS 16

static int g_bvh_method = -1; /* -1 auto (PLOC for render scenes, Karras for filter scenes), 0 PLOC, 1 Karras */
void orc_set_bvh_method(int method) { g_bvh_method = method == 1 ? 1 : (method == 0 ? 0 : -1); }
int orc_get_bvh_method(void) { return g_bvh_method; }
static int bvh_method_for(int filterScene) { return g_bvh_method >= 0 ? g_bvh_method : (filterScene ? 1 : 0); }

static float union_area(const float* al, const float* ah, const float* bl, const float* bh) {
  float dx = fmaxf(ah[0], bh[0]) - fminf(al[0], bl[0]);
  float dy = fmaxf(ah[1], bh[1]) - fminf(al[1], bl[1]);
  float dz = fmaxf(ah[2], bh[2]) - fminf(al[2], bl[2]);
  return dx * dy + dy * dz + dz * dx;
}

typedef struct {
  int *left, *right, *parent, *leafParent, *count, *height, *collapse, *first, *leafPos;
  float *lo, *hi, *cost; /* 4 floats per box */
} ploc_t;

/* A new inner node nd over clusters a and b (boxes al/ah, bl/bh): box, SAH
 * cost, primitive count, height and the leaf-collapse decision, in the
 * kernel's float operation order (make_node). */
static void ploc_node(ploc_t* P, int nd, int a, const float* al, const float* ah, int b, const float* bl,
                      const float* bh) {
  float ca = a < 0 ? SAH_TRI : P->cost[a], cb = b < 0 ? SAH_TRI : P->cost[b];
  int na = a < 0 ? 1 : P->count[a], nb = b < 0 ? 1 : P->count[b];
  int ha = a < 0 ? 0 : P->height[a], hb = b < 0 ? 0 : P->height[b];
  float* lo = &P->lo[4 * (size_t)nd];
  float* hi = &P->hi[4 * (size_t)nd];
  for (int k = 0; k < 3; ++k) {
    lo[k] = fminf(al[k], bl[k]);
    hi[k] = fmaxf(ah[k], bh[k]);
  }
  lo[3] = hi[3] = 0.0f;
  float A = box_area(lo, hi), Al = box_area(al, ah), Ar = box_area(bl, bh);
  float inner = (A > 0.0f) ? SAH_NODE + (Al * ca + Ar * cb) / A : SAH_NODE + ca + cb;
  int count = na + nb;
  float leafc = SAH_TRI * (float)count;
  int col = (count <= LEAF_MAX && leafc <= inner) ? 1 : 0;
  P->left[nd] = a;
  P->right[nd] = b;
  P->cost[nd] = col ? leafc : inner;
  P->count[nd] = count;
  P->height[nd] = col ? 0 : 1 + (ha > hb ? ha : hb);
  P->collapse[nd] = col;
  if (a < 0) P->leafParent[~a] = nd; else P->parent[a] = nd;
  if (b < 0) P->leafParent[~b] = nd; else P->parent[b] = nd;
}

/* Clustering of the n >= 2 sorted leaves (boxes leafLo/leafHi): each
 * iteration every cluster finds its nearest neighbour within PLOC_RADIUS
 * positions (smallest enclosing area; then closest position, even lower
 * position, lower position — the GPU's 64-bit pair key), mutual pairs
 * merge into a node at the smaller position (numbered downwards from n-2 in
 * position order), the list is compacted.  Then depth-first positions of the
 * leaves and the first position of every node. */
static void ploc_build(ploc_t* P, int n, const float* leafLo, const float* leafHi) {
  int* ref = (int*)malloc(sizeof(int) * (size_t)n);
  int* ref2 = (int*)malloc(sizeof(int) * (size_t)n);
  float* lo = (float*)malloc(sizeof(float) * 4 * (size_t)n);
  float* hi = (float*)malloc(sizeof(float) * 4 * (size_t)n);
  float* lo2 = (float*)malloc(sizeof(float) * 4 * (size_t)n);
  float* hi2 = (float*)malloc(sizeof(float) * 4 * (size_t)n);
  int* nn = (int*)malloc(sizeof(int) * (size_t)n);
  for (int i = 0; i < n; ++i) ref[i] = ~i;
  memcpy(lo, leafLo, sizeof(float) * 4 * (size_t)n);
  memcpy(hi, leafHi, sizeof(float) * 4 * (size_t)n);
  for (int i = 0; i < n - 1; ++i) P->parent[i] = -1;
  int m = n, cursor = n - 1;
  while (m > 1) {
    for (int i = 0; i < m; ++i) {
      int j0 = i - PLOC_RADIUS < 0 ? 0 : i - PLOC_RADIUS, j1 = i + PLOC_RADIUS > m - 1 ? m - 1 : i + PLOC_RADIUS;
      uint64_t best = UINT64_MAX;
      for (int j = j0; j <= j1; ++j) {
        if (j == i) continue;
        float a = union_area(&lo[4 * (size_t)i], &hi[4 * (size_t)i], &lo[4 * (size_t)j], &hi[4 * (size_t)j]);
        uint32_t ab;
        memcpy(&ab, &a, 4);
        uint32_t d = (uint32_t)(i > j ? i - j : j - i), lo2 = (uint32_t)(i < j ? i : j);
        uint64_t key = ((uint64_t)ab << 32) | ((uint64_t)d << 27) | ((uint64_t)(lo2 & 1u) << 26) | lo2;
        if (key < best) best = key;
      }
      int blo = (int)(best & 0x03FFFFFFu), bd = (int)((best >> 27) & 31u);
      nn[i] = blo < i ? blo : i + bd;
    }
    int k = 0;
    for (int i = 0; i < m; ++i)
      if (nn[nn[i]] == i && i < nn[i]) ++k;
    int base = cursor - k, rank = 0, pos = 0;
    for (int i = 0; i < m; ++i) {
      int j = nn[i];
      int mutual = nn[j] == i;
      if (mutual && j < i) continue;
      if (mutual) {
        int nd = base + rank++;
        ploc_node(P, nd, ref[i], &lo[4 * (size_t)i], &hi[4 * (size_t)i], ref[j], &lo[4 * (size_t)j],
                  &hi[4 * (size_t)j]);
        ref2[pos] = nd;
        memcpy(&lo2[4 * (size_t)pos], &P->lo[4 * (size_t)nd], 16);
        memcpy(&hi2[4 * (size_t)pos], &P->hi[4 * (size_t)nd], 16);
      } else {
        ref2[pos] = ref[i];
        memcpy(&lo2[4 * (size_t)pos], &lo[4 * (size_t)i], 16);
        memcpy(&hi2[4 * (size_t)pos], &hi[4 * (size_t)i], 16);
      }
      ++pos;
    }
    cursor = base;
    m = pos;
    int* tr = ref; ref = ref2; ref2 = tr;
    float* tl = lo; lo = lo2; lo2 = tl;
    float* th = hi; hi = hi2; hi2 = th;
  }
  for (int i = 0; i < n; ++i) {
    int cur = ~i, p = P->leafParent[i], pos = 0;
    while (p >= 0) {
      if (P->right[p] == cur) pos += P->left[p] < 0 ? 1 : P->count[P->left[p]];
      cur = p;
      p = P->parent[p];
    }
    P->leafPos[i] = pos;
    cur = ~i;
    p = P->leafParent[i];
    while (p >= 0 && P->left[p] == cur) {
      P->first[p] = pos;
      cur = p;
      p = P->parent[p];
    }
  }
  free(ref); free(ref2); free(lo); free(hi); free(lo2); free(hi2); free(nn);
}

static int ploc_child_ref(const ploc_t* P, int c) {
  if (c < 0) return ~(P->leafPos[~c] | (1 << 26));
  if (P->collapse[c]) return ~(P->first[c] | (P->count[c] << 26));
  return c;
}

static int build_bvh_impl(const float* pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris, int32_t* nodes_out,
                          uint32_t* order_out, float* tris_out, int method);

int orc_build_bvh(const float* pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris, int32_t* nodes_out,
                  uint32_t* order_out, float* tris_out) {
  return build_bvh_impl(pos, nverts, idx, ntris, nodes_out, order_out, tris_out, bvh_method_for(0));
}

int orc_build_bvh_filter(const float* pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris, int32_t* nodes_out,
                         uint32_t* order_out, float* tris_out) {
  return build_bvh_impl(pos, nverts, idx, ntris, nodes_out, order_out, tris_out, bvh_method_for(1));
}

static int build_bvh_impl(const float* pos, uint32_t nverts, const uint32_t* idx, uint32_t ntris, int32_t* nodes_out,
                          uint32_t* order_out, float* tris_out, int method) {
  (void)nverts;
  if (ntris == 0 || ntris >= (1u << 26)) return -1;
  int n = (int)ntris;
  float* tlo = (float*)malloc(sizeof(float) * 4 * (size_t)n);
  float* thi = (float*)malloc(sizeof(float) * 4 * (size_t)n);
  float cmin[3] = {INFINITY, INFINITY, INFINITY}, cmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int t = 0; t < n; ++t) {
    const uint32_t* tv = &idx[3 * (size_t)t];
    for (int k = 0; k < 3; ++k) {
      float a = pos[3 * (size_t)tv[0] + k], b = pos[3 * (size_t)tv[1] + k], c = pos[3 * (size_t)tv[2] + k];
      float l = fminf(fminf(a, b), c), h = fmaxf(fmaxf(a, b), c);
      tlo[4 * t + k] = l;
      thi[4 * t + k] = h;
      float cen = (l + h) * 0.5f;
      cmin[k] = fminf(cmin[k], cen);
      cmax[k] = fmaxf(cmax[k], cen);
    }
    tlo[4 * t + 3] = thi[4 * t + 3] = 0.0f;
  }
  float inv[3];
  for (int k = 0; k < 3; ++k) {
    float e = cmax[k] - cmin[k];
    inv[k] = e > 0.0f ? 1.0f / e : 0.0f;
  }
  kv_t* kv = (kv_t*)malloc(sizeof(kv_t) * (size_t)n);
  for (int t = 0; t < n; ++t) {
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
      float cen = (tlo[4 * t + k] + thi[4 * t + k]) * 0.5f;
      q[k] = quant21(cen, cmin[k], inv[k]);
    }
    kv[t].key = (expand21(q[0]) << 2) | (expand21(q[1]) << 1) | expand21(q[2]);
    kv[t].idx = (uint32_t)t;
  }
  qsort(kv, (size_t)n, sizeof(kv_t), kv_cmp);
  uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  for (int i = 0; i < n; ++i) {
    keys[i] = kv[i].key;
    order_out[i] = kv[i].idx;
  }
  int plocHeight = -1;
  if (n > 1 && method == 0) {
    int ni = n - 1;
    ploc_t P;
    P.left = (int*)malloc(sizeof(int) * ni); P.right = (int*)malloc(sizeof(int) * ni);
    P.parent = (int*)malloc(sizeof(int) * ni); P.leafParent = (int*)malloc(sizeof(int) * (size_t)n);
    P.count = (int*)malloc(sizeof(int) * ni); P.height = (int*)malloc(sizeof(int) * ni);
    P.collapse = (int*)malloc(sizeof(int) * ni); P.first = (int*)malloc(sizeof(int) * ni);
    P.leafPos = (int*)malloc(sizeof(int) * (size_t)n);
    P.lo = (float*)malloc(sizeof(float) * 4 * ni); P.hi = (float*)malloc(sizeof(float) * 4 * ni);
    P.cost = (float*)malloc(sizeof(float) * ni);
    float* sLo = (float*)malloc(sizeof(float) * 4 * (size_t)n);
    float* sHi = (float*)malloc(sizeof(float) * 4 * (size_t)n);
    uint32_t* sorted = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    for (int i = 0; i < n; ++i) {
      sorted[i] = order_out[i];
      memcpy(&sLo[4 * (size_t)i], &tlo[4 * (size_t)sorted[i]], 16);
      memcpy(&sHi[4 * (size_t)i], &thi[4 * (size_t)sorted[i]], 16);
    }
    ploc_build(&P, n, sLo, sHi);
    for (int i = 0; i < n; ++i) order_out[P.leafPos[i]] = sorted[i];
    for (int i = 0; i < ni; ++i) {
      int32_t* w = &nodes_out[16 * (size_t)i];
      memset(w, 0, 64);
      if (i == 0 && P.collapse[0]) {
        float el[3] = {INFINITY, INFINITY, INFINITY}, eh[3] = {-INFINITY, -INFINITY, -INFINITY};
        put_box(w, 0, &P.lo[0], &P.hi[0]);
        put_box(w, 1, el, eh);
        w[12] = leaf_ref(0, n);
        w[13] = BVH_NONE;
        w[14] = -1;
        w[15] = 0;
        continue;
      }
      int lc = P.left[i], rc = P.right[i];
      put_box(w, 0, lc < 0 ? &sLo[4 * (size_t)(~lc)] : &P.lo[4 * (size_t)lc],
              lc < 0 ? &sHi[4 * (size_t)(~lc)] : &P.hi[4 * (size_t)lc]);
      put_box(w, 1, rc < 0 ? &sLo[4 * (size_t)(~rc)] : &P.lo[4 * (size_t)rc],
              rc < 0 ? &sHi[4 * (size_t)(~rc)] : &P.hi[4 * (size_t)rc]);
      w[12] = ploc_child_ref(&P, lc);
      w[13] = ploc_child_ref(&P, rc);
      w[14] = P.parent[i];
      w[15] = P.height[i];
    }
    plocHeight = P.collapse[0] ? 1 : P.height[0];
    free(P.left); free(P.right); free(P.parent); free(P.leafParent); free(P.count); free(P.height);
    free(P.collapse); free(P.first); free(P.leafPos); free(P.lo); free(P.hi); free(P.cost);
    free(sLo); free(sHi); free(sorted);
  }
  if (tris_out) {
    for (int i = 0; i < n; ++i) {
      uint32_t p = order_out[i];
      for (int v = 0; v < 3; ++v) {
        uint32_t vi = idx[3 * (size_t)p + v];
        tris_out[12 * (size_t)i + 4 * v + 0] = pos[3 * (size_t)vi];
        tris_out[12 * (size_t)i + 4 * v + 1] = pos[3 * (size_t)vi + 1];
        tris_out[12 * (size_t)i + 4 * v + 2] = pos[3 * (size_t)vi + 2];
        float w = 0.0f;
        if (v == 0) memcpy(&w, &p, 4);
        tris_out[12 * (size_t)i + 4 * v + 3] = w;
      }
    }
  }
  int height = 0;
  if (plocHeight >= 0) {
    height = plocHeight;
  } else if (n == 1) {
    int32_t* w = nodes_out;
    memset(w, 0, 64);
    float el[3] = {INFINITY, INFINITY, INFINITY}, eh[3] = {-INFINITY, -INFINITY, -INFINITY};
    put_box(w, 0, &tlo[0], &thi[0]);
    put_box(w, 1, el, eh);
    w[12] = leaf_ref(0, 1);
    w[13] = BVH_NONE;
    w[14] = -1;
    w[15] = 0;
    height = 1;
  } else {
    int ni = n - 1;
    bld_t B;
    B.n = n;
    B.left = (int*)malloc(sizeof(int) * ni);
    B.right = (int*)malloc(sizeof(int) * ni);
    B.first = (int*)malloc(sizeof(int) * ni);
    B.last = (int*)malloc(sizeof(int) * ni);
    B.parent = (int*)malloc(sizeof(int) * ni);
    B.collapse = (int*)malloc(sizeof(int) * ni);
    B.height = (int*)malloc(sizeof(int) * ni);
    B.lo = (float*)malloc(sizeof(float) * 4 * ni);
    B.hi = (float*)malloc(sizeof(float) * 4 * ni);
    B.cost = (float*)malloc(sizeof(float) * ni);
    B.leafLo = (float*)malloc(sizeof(float) * 4 * (size_t)n);
    B.leafHi = (float*)malloc(sizeof(float) * 4 * (size_t)n);
    for (int i = 0; i < n; ++i) {
      memcpy(&B.leafLo[4 * i], &tlo[4 * (size_t)order_out[i]], 16);
      memcpy(&B.leafHi[4 * i], &thi[4 * (size_t)order_out[i]], 16);
    }
    B.parent[0] = -1;
    for (int i = 0; i < ni; ++i) {
      int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
      int dmin = kdelta(keys, n, i, i - d);
      int lmax = 2;
      while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
      int l = 0;
      for (int t = lmax / 2; t >= 1; t /= 2)
        if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
      int j = i + l * d;
      int dnode = kdelta(keys, n, i, j);
      int s = 0, div = 2;
      int t = (l + div - 1) / div;
      for (;;) {
        if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
        div *= 2;
        t = (l + div - 1) / div;
      }
      int gamma = i + s * d + (d < 0 ? -1 : 0);
      int f = i < j ? i : j, la = i < j ? j : i;
      B.left[i] = (f == gamma) ? ~gamma : gamma;
      B.right[i] = (la == gamma + 1) ? ~(gamma + 1) : (gamma + 1);
      B.first[i] = f;
      B.last[i] = la;
      if (B.left[i] >= 0) B.parent[B.left[i]] = i;
      if (B.right[i] >= 0) B.parent[B.right[i]] = i;
    }
    bottom_up(&B, 0);
    for (int i = 0; i < ni; ++i) {
      int32_t* w = &nodes_out[16 * (size_t)i];
      memset(w, 0, 64);
      if (i == 0 && B.collapse[0]) {
        float el[3] = {INFINITY, INFINITY, INFINITY}, eh[3] = {-INFINITY, -INFINITY, -INFINITY};
        put_box(w, 0, &B.lo[0], &B.hi[0]);
        put_box(w, 1, el, eh);
        w[12] = leaf_ref(0, n);
        w[13] = BVH_NONE;
        w[14] = -1;
        w[15] = 0;
        continue;
      }
      int lc = B.left[i], rc = B.right[i];
      put_box(w, 0, lc < 0 ? &B.leafLo[4 * (~lc)] : &B.lo[4 * lc], lc < 0 ? &B.leafHi[4 * (~lc)] : &B.hi[4 * lc]);
      put_box(w, 1, rc < 0 ? &B.leafLo[4 * (~rc)] : &B.lo[4 * rc], rc < 0 ? &B.leafHi[4 * (~rc)] : &B.hi[4 * rc]);
      w[12] = child_ref(&B, lc);
      w[13] = child_ref(&B, rc);
      w[14] = B.parent[i];
      w[15] = B.height[i];
    }
    height = B.collapse[0] ? 1 : B.height[0];
    free(B.left); free(B.right); free(B.first); free(B.last); free(B.parent); free(B.collapse);
    free(B.height); free(B.lo); free(B.hi); free(B.cost); free(B.leafLo); free(B.leafHi);
  }
  free(tlo); free(thi); free(kv); free(keys);
  return height;
}

/* ---------------------------------------------------------------- traversal */

typedef struct {
  f3 o, d, invd;
  int kx, ky, kz;
  float Sx, Sy, Sz;
} rpre_t;

static rpre_t make_pre(f3 o, f3 d) {
  rpre_t r;
  r.o = o;
  r.d = d;
  r.invd = F3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
  int kx = kz + 1; if (kx == 3) kx = 0;
  int ky = kx + 1; if (ky == 3) ky = 0;
  if (comp3(d, kz) < 0.0f) { int t = kx; kx = ky; ky = t; }
  r.kx = kx; r.ky = ky; r.kz = kz;
  float dz = comp3(d, kz);
  r.Sx = comp3(d, kx) / dz;
  r.Sy = comp3(d, ky) / dz;
  r.Sz = 1.0f / dz;
  return r;
}

static int slab(const rpre_t* r, const float* b, int slot, float tmax, float* tentry) {
  float lox, hix, loy, hiy, loz, hiz;
  if (slot == 0) { lox = b[0]; hix = b[1]; loy = b[2]; hiy = b[3]; loz = b[8]; hiz = b[9]; }
  else { lox = b[4]; hix = b[5]; loy = b[6]; hiy = b[7]; loz = b[10]; hiz = b[11]; }
  float tx0 = (lox - r->o.x) * r->invd.x, tx1 = (hix - r->o.x) * r->invd.x;
  float ty0 = (loy - r->o.y) * r->invd.y, ty1 = (hiy - r->o.y) * r->invd.y;
  float tz0 = (loz - r->o.z) * r->invd.z, tz1 = (hiz - r->o.z) * r->invd.z;
  float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
  float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
  tf = tf * 1.00000024f;
  *tentry = tn;
  return tn <= tf;
}


void oi_tex_lookup(const oi_tex* t, float u, float v, float out[4]) {
  u = u - floorf(u);
  v = v - floorf(v);
  const float xb = u * (float)t->W - 0.5f, yb = v * (float)t->H - 0.5f;
  const float fx = floorf(xb), fy = floorf(yb);
  const float a = xb - fx, b = yb - fy;
  const int x0 = (int)fx, y0 = (int)fy;
  const float* tx[4];
  for (int k = 0; k < 4; ++k) {
    int x = x0 + (k & 1), y = y0 + (k >> 1);
    x %= t->W;
    if (x < 0) x += t->W;
    y %= t->H;
    if (y < 0) y += t->H;
    tx[k] = &t->texels[4 * ((size_t)y * t->W + x)];
  }
  const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
  for (int c = 0; c < 4; ++c) out[c] = w00 * tx[0][c] + w10 * tx[1][c] + w01 * tx[2][c] + w11 * tx[3][c];
}

void oi_tex_from(const orc_texture* src, int kind, oi_tex* t) {
  t->W = (int)src->width;
  t->H = (int)src->height;
  const size_t n = (size_t)t->W * t->H;
  t->texels = (float*)malloc(sizeof(float) * 4 * n);
  for (size_t i = 0; i < n; ++i) {
    const uint8_t* p = &src->rgba[4 * i];
    const float r = (float)p[0] / 255.0f, g = (float)p[1] / 255.0f, b = (float)p[2] / 255.0f;
    float* o = &t->texels[4 * i];
    if (kind == OI_TEX_ALPHA) {
      const float a = (float)p[3] / 255.0f;
      o[0] = o[1] = o[2] = a;
    } else if (kind == OI_TEX_LUMA) {
      float l = 0.2126f * r;
      l += 0.7152f * g;
      l += 0.0722f * b;
      o[0] = o[1] = o[2] = l;
    } else {
      o[0] = r; o[1] = g; o[2] = b;
    }
    o[3] = 1.0f;
  }
}

void oi_material_maps(const orc_material* m, const orc_texture* albedo, const orc_texture* specular,
                      const orc_texture* normal, const orc_texture* alpha, oi_tex* tex, int* ntex, int out[4]) {
  for (int k = 0; k < 4; ++k) out[k] = -1;
  const float* ks = m->specular;
  if (albedo) { oi_tex_from(albedo, OI_TEX_COLOR, &tex[*ntex]); out[0] = (*ntex)++; }
  if (albedo && (ks[0] <= 0.02f || ks[1] <= 0.02f || ks[2] <= 0.02f)) {
    oi_tex_from(albedo, OI_TEX_LUMA, &tex[*ntex]); out[1] = (*ntex)++;
  } else if (specular) {
    oi_tex_from(specular, OI_TEX_COLOR, &tex[*ntex]); out[1] = (*ntex)++;
  }
  if (normal) { oi_tex_from(normal, OI_TEX_COLOR, &tex[*ntex]); out[2] = (*ntex)++; }
  if (alpha) { oi_tex_from(alpha, OI_TEX_COLOR, &tex[*ntex]); out[3] = (*ntex)++; }
  else if (albedo && albedo->channels == 4) { oi_tex_from(albedo, OI_TEX_ALPHA, &tex[*ntex]); out[3] = (*ntex)++; }
}

void oi_textured_surface(const oi_tex* tex, int tAlbedo, int tGlossy, int tNormal, const float* uv,
                         const float* tv, float b1, float b2, f3* n, f3* diffuse, f3* specular) {
  const float b0 = (1.0f - b1) - b2;
  const float tcx = b0 * uv[0] + b1 * uv[2] + b2 * uv[4], tcy = b0 * uv[1] + b1 * uv[3] + b2 * uv[5];
  float c[4];
  if (tAlbedo >= 0) {
    oi_tex_lookup(&tex[tAlbedo], tcx, tcy, c);
    *diffuse = F3(c[0], c[1], c[2]);
  }
  if (tGlossy >= 0) {
    oi_tex_lookup(&tex[tGlossy], tcx, tcy, c);
    *specular = F3(c[0], c[1], c[2]);
  }
  if (tNormal >= 0) {
    const f3 P0 = F3(tv[0], tv[1], tv[2]), P1 = F3(tv[4], tv[5], tv[6]), P2 = F3(tv[8], tv[9], tv[10]);
    const f3 P = add3(add3(mul3s(P0, b0), mul3s(P1, b1)), mul3s(P2, b2));
    const f3 e1 = sub3(P1, P), e2 = sub3(P2, P);
    const float du1 = uv[2] - tcx, dv1 = uv[3] - tcy, du2 = uv[4] - tcx, dv2 = uv[5] - tcy;
    const float den = du1 * dv2 - du2 * dv1;
    if (den != 0.0f) {
      const float f = 1.0f / den;
      const f3 T = F3(f * (dv2 * e1.x - dv1 * e2.x), f * (dv2 * e1.y - dv1 * e2.y), f * (dv2 * e1.z - dv1 * e2.z));
      const f3 B = F3(f * (-du2 * e1.x + du1 * e2.x), f * (-du2 * e1.y + du1 * e2.y), f * (-du2 * e1.z + du1 * e2.z));
      const int tz = T.x == 0.0f && T.y == 0.0f && T.z == 0.0f, bz = B.x == 0.0f && B.y == 0.0f && B.z == 0.0f;
      if (!tz && !bz) {
        oi_tex_lookup(&tex[tNormal], tcx, tcy, c);
        const f3 nt = F3(c[0] * 2.0f - 1.0f, c[1] * 2.0f - 1.0f, c[2] * 2.0f - 1.0f);
        if (!(nt.x == 0.0f && nt.y == 0.0f && nt.z == 0.0f)) {
          const f3 v = norm3(nt);
          *n = norm3(add3(add3(mul3s(norm3(T), v.x), mul3s(norm3(neg3(B)), v.y)), mul3s(*n, v.z)));
        }
      }
    }
  }
}

static int alpha_opaque(const oi_alpha* a, int tri, float b1, float b2) {
  const int k = a->alpha_tex[tri];
  if (k < 0) return 1;
  const float* uv = &a->uv[6 * (size_t)tri];
  const float b0 = (1.0f - b1) - b2;
  const float u = b0 * uv[0] + b1 * uv[2] + b2 * uv[4], v = b0 * uv[1] + b1 * uv[3] + b2 * uv[5];
  float c[4];
  oi_tex_lookup(&a->tex[k], u, v, c);
  return c[0] > 0.0f;
}

static int tri_test(const rpre_t* r, f3 p0, f3 p1, f3 p2, int tri, hit_t* best, const oi_alpha* alpha) {
  f3 A = sub3(p0, r->o), B = sub3(p1, r->o), C = sub3(p2, r->o);
  float Az0 = comp3(A, r->kz), Bz0 = comp3(B, r->kz), Cz0 = comp3(C, r->kz);
  float Ax = comp3(A, r->kx) - r->Sx * Az0, Ay = comp3(A, r->ky) - r->Sy * Az0;
  float Bx = comp3(B, r->kx) - r->Sx * Bz0, By = comp3(B, r->ky) - r->Sy * Bz0;
  float Cx = comp3(C, r->kx) - r->Sx * Cz0, Cy = comp3(C, r->ky) - r->Sy * Cz0;
  float U = Cx * By - Cy * Bx;
  float V = Ax * Cy - Ay * Cx;
  float W = Bx * Ay - By * Ax;
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    double CxBy = (double)Cx * (double)By, CyBx = (double)Cy * (double)Bx;
    U = (float)(CxBy - CyBx);
    double AxCy = (double)Ax * (double)Cy, AyCx = (double)Ay * (double)Cx;
    V = (float)(AxCy - AyCx);
    double BxAy = (double)Bx * (double)Ay, ByAx = (double)By * (double)Ax;
    W = (float)(BxAy - ByAx);
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return 0;
  float det = U + V + W;
  if (det == 0.0f) return 0;
  float Az = r->Sz * Az0, Bz = r->Sz * Bz0, Cz = r->Sz * Cz0;
  float T = U * Az + V * Bz + W * Cz;
  float rcp = 1.0f / det;
  float t = T * rcp;
  if (!(t > 0.0f)) return 0;
  if (t < best->t || (t == best->t && tri < best->tri)) {
    const float b1 = V * rcp, b2 = W * rcp;
    if (alpha && !alpha_opaque(alpha, tri, b1, b2)) return 0;
    best->t = t;
    best->b1 = b1;
    best->b2 = b2;
    best->tri = tri;
    return 1;
  }
  return 0;
}

hit_t oi_trace(const int32_t* nodes, const float* tris, f3 o, f3 d, float tmax, int any_hit) {
  return oi_trace_alpha(nodes, tris, o, d, tmax, any_hit, NULL);
}

hit_t oi_trace_alpha(const int32_t* nodes, const float* tris, f3 o, f3 d, float tmax, int any_hit,
                     const oi_alpha* alpha) {
  hit_t best;
  best.t = tmax;
  best.b1 = best.b2 = 0.0f;
  best.tri = 0x7FFFFFFF;
  rpre_t r = make_pre(o, d);
  int stack[BVH_STACK];
  float stackT[BVH_STACK];
  int sp = 0, cur = 0, found = 0;
  for (;;) {
    if (cur >= 0) {
      const int32_t* w = &nodes[16 * (size_t)cur];
      const float* b = (const float*)w;
      float t0 = 0.0f, t1 = 0.0f;
      int h0 = slab(&r, b, 0, best.t, &t0);
      int h1 = (w[13] != BVH_NONE) && slab(&r, b, 1, best.t, &t1);
      if (h0 && h1) {
        int nearC = w[12], farC = w[13];
        float farT = t1;
        if (t1 < t0) { nearC = w[13]; farC = w[12]; farT = t0; }
        stack[sp] = farC;
        stackT[sp] = farT;
        ++sp;
        cur = nearC;
        continue;
      } else if (h0) { cur = w[12]; continue; }
      else if (h1) { cur = w[13]; continue; }
    } else {
      int first = (~cur) & 0x03FFFFFF, count = ((~cur) >> 26) & 0x1F;
      for (int i = 0; i < count; ++i) {
        int tri = first + i;
        const float* tv = &tris[12 * (size_t)tri];
        if (tri_test(&r, F3(tv[0], tv[1], tv[2]), F3(tv[4], tv[5], tv[6]), F3(tv[8], tv[9], tv[10]), tri, &best,
                     alpha)) {
          found = 1;
          if (any_hit) return best;
        }
      }
    }
    for (;;) {
      if (sp == 0) {
        if (!found) best.tri = -1;
        return best;
      }
      --sp;
      if (stackT[sp] <= best.t) break;
    }
    cur = stack[sp];
  }
}

int orc_trace(const int32_t* nodes, const float* tris, float ox, float oy, float oz, float dx, float dy, float dz,
              float tmax, float* t, float* b1, float* b2) {
  hit_t h = oi_trace(nodes, tris, F3(ox, oy, oz), F3(dx, dy, dz), tmax, 0);
  *t = h.t;
  *b1 = h.b1;
  *b2 = h.b2;
  return h.tri;
}

/* ---------------------------------------------------------------- grid setup */


m4_t oi_m4_id(void) {
  m4_t r;
  memset(&r, 0, sizeof(r));
  for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0f;
  return r;
}
m4_t oi_m4_mul(m4_t a, m4_t b) {
  m4_t r;
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i) {
      float v = a.m[0][i] * b.m[j][0];
      v = v + a.m[1][i] * b.m[j][1];
      v = v + a.m[2][i] * b.m[j][2];
      v = v + a.m[3][i] * b.m[j][3];
      r.m[j][i] = v;
    }
  return r;
}
m4_t oi_m4_inv(m4_t a) {
  double A[4][8];
  for (int r = 0; r < 4; ++r) {
    for (int c = 0; c < 4; ++c) A[r][c] = a.m[c][r];
    for (int c = 0; c < 4; ++c) A[r][4 + c] = (r == c) ? 1.0 : 0.0;
  }
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    for (int r = c + 1; r < 4; ++r)
      if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
    if (piv != c)
      for (int k = 0; k < 8; ++k) { double t = A[c][k]; A[c][k] = A[piv][k]; A[piv][k] = t; }
    double p = A[c][c];
    if (p == 0.0) return oi_m4_id();
    for (int k = 0; k < 8; ++k) A[c][k] /= p;
    for (int r = 0; r < 4; ++r) {
      if (r == c) continue;
      double f = A[r][c];
      if (f == 0.0) continue;
      for (int k = 0; k < 8; ++k) A[r][k] -= f * A[c][k];
    }
  }
  m4_t o;
  for (int row = 0; row < 4; ++row)
    for (int c = 0; c < 4; ++c) o.m[c][row] = (float)A[row][4 + c];
  return o;
}
static m4_t m4_from43(const float* f) {
  m4_t r;
  for (int c = 0; c < 4; ++c) {
    r.m[c][0] = f[3 * c]; r.m[c][1] = f[3 * c + 1]; r.m[c][2] = f[3 * c + 2];
    r.m[c][3] = c == 3 ? 1.0f : 0.0f;
  }
  return r;
}
void oi_m4_to43(m4_t a, float* f) {
  for (int c = 0; c < 4; ++c) { f[3 * c] = a.m[c][0]; f[3 * c + 1] = a.m[c][1]; f[3 * c + 2] = a.m[c][2]; }
}

void orc_setup_grid(const float* mlo, const float* mhi, const float* m2w, float vs, orc_grid* g) {
  memset(g, 0, sizeof(*g));
  /* SAABB::transform of the object's model box: min and max corners only */
  f3 a = xpoint(m2w, F3(mlo[0], mlo[1], mlo[2])), b = xpoint(m2w, F3(mhi[0], mhi[1], mhi[2]));
  f3 wlo = F3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z));
  f3 whi = F3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z));
  m4_t w2m = oi_m4_inv(m4_from43(m2w));
  f3 ext = sub3(whi, wlo);
  int nv[3] = {(int)ceilf(ext.x / vs - 0.001f), (int)ceilf(ext.y / vs - 0.001f), (int)ceilf(ext.z / vs - 0.001f)};
  for (int k = 0; k < 3; ++k) g->num_voxels[k] = nv[k];
  m4_t T = oi_m4_id(), S1 = oi_m4_id(), S2 = oi_m4_id();
  T.m[3][0] = wlo.x; T.m[3][1] = wlo.y; T.m[3][2] = wlo.z;
  S1.m[0][0] = ext.x; S1.m[1][1] = ext.y; S1.m[2][2] = ext.z;
  S2.m[0][0] = 1.0f / (float)nv[0]; S2.m[1][1] = 1.0f / (float)nv[1]; S2.m[2][2] = 1.0f / (float)nv[2];
  m4_t i2m = oi_m4_mul(oi_m4_mul(oi_m4_mul(w2m, T), S1), S2);
  m4_t m2i = oi_m4_inv(i2m);
  m4_t m2wI = oi_m4_inv(w2m);
  m4_t i2w = oi_m4_mul(m2wI, i2m);
  float i2w43[12];
  oi_m4_to43(i2w, i2w43);
  f3 p0 = xpoint(i2w43, F3(0.0f, 0.0f, 0.0f));
  f3 p1 = xpoint(i2w43, F3((float)nv[0], (float)nv[1], (float)nv[2]));
  g->world_bb_min[0] = fminf(p0.x, p1.x); g->world_bb_min[1] = fminf(p0.y, p1.y); g->world_bb_min[2] = fminf(p0.z, p1.z);
  g->world_bb_max[0] = fmaxf(p0.x, p1.x); g->world_bb_max[1] = fmaxf(p0.y, p1.y); g->world_bb_max[2] = fmaxf(p0.z, p1.z);
  oi_m4_to43(i2m, g->index_to_model);
  oi_m4_to43(m2i, g->model_to_index);
  oi_m4_to43(m2wI, g->model_to_world);
  oi_m4_to43(w2m, g->world_to_model);
  g->voxel_size = vs;
}

/* ---------------------------------------------------------------- filter */

/* Sphere::intersect for an origin inside the sphere: the far root. */
static float sphere_exit(f3 o, f3 d, f3 c, float radius) {
  f3 oc = sub3(o, c);
  float a = dot3(d, d);
  float b = 2.0f * dot3(d, oc);
  float cc = dot3(oc, oc) - radius * radius;
  float disc = b * b - 4.0f * a * cc;
  if (disc == 0.0f) {
    float t = (-b + sqrtf(disc)) / (2.0f * a);
    return t > 0.0f ? t : 0.0f;
  }
  if (disc > 0.0f) {
    float sq = sqrtf(disc);
    float den = 1.0f / (2.0f * a);
    float t1 = (-b + sq) * den, t2 = (-b - sq) * den;
    float mn = fminf(t1, t2), mx = fmaxf(t1, t2);
    if (mx > 0.0f) return mn > 0.0f ? mn : mx;
  }
  return 0.0f;
}

static uint16_t q16(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 65535.0) return 65535;
  return (uint16_t)v;
}
static uint8_t q8(double v) {
  if (!(v > 0.0)) return 0;
  if (v >= 255.0) return 255;
  return (uint8_t)v;
}
static double clampd(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

uint16_t oi_half_bits(float f) {
  uint32_t x;
  memcpy(&x, &f, 4);
  uint32_t sign = (x >> 16) & 0x8000u, mag = x & 0x7FFFFFFFu;
  if (mag >= 0x7F800000u) return (uint16_t)(sign | 0x7C00u | (mag > 0x7F800000u ? 0x200u : 0u));
  if (mag >= 0x477FF000u) return (uint16_t)(sign | 0x7C00u);
  if (mag < 0x38800000u) {
    if (mag < 0x33000000u) return (uint16_t)sign;
    uint32_t e = mag >> 23, m = (mag & 0x7FFFFFu) | 0x800000u, shift = 126u - e;
    uint32_t v = m >> shift, rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1u);
    if (rem > half || (rem == half && (v & 1u))) ++v;
    return (uint16_t)(sign | v);
  }
  uint32_t v = (mag - 0x38000000u) >> 13, rem = mag & 0x1FFFu;
  if (rem > 0x1000u || (rem == 0x1000u && (v & 1u))) ++v;
  return (uint16_t)(sign | v);
}

void orc_encode(const double* w, uint8_t* out) {
  const double M16 = 65535.0, M8 = 255.0;
  memset(out, 0, 32);
  float density = (float)w[0];
  memcpy(out, &density, 4);
  double sxx = w[1], syy = w[2], szz = w[3], sxy = w[4], sxz = w[5], syz = w[6];
  uint16_t u[6];
  u[0] = q16(clampd(M16 * sqrt(sxx), 0.0, M16));
  u[1] = q16(clampd(M16 * sqrt(syy), 0.0, M16));
  u[2] = q16(clampd(M16 * sqrt(szz), 0.0, M16));
  u[3] = q16(clampd(M16 * 0.5 * (sxy / sqrt(sxx * syy) + 1.0), 0.0, M16));
  u[4] = q16(clampd(M16 * 0.5 * (sxz / sqrt(sxx * szz) + 1.0), 0.0, M16));
  u[5] = q16(clampd(M16 * 0.5 * (syz / sqrt(syy * szz) + 1.0), 0.0, M16));
  memcpy(out + 4, u, 12);
  for (int k = 0; k < 3; ++k) {
    out[16 + k] = q8(clampd(M8 * w[7 + k], 0.0, M8));
    out[19 + k] = q8(clampd(M8 * w[10 + k], 0.0, M8));
  }
  double nl = sqrt(w[13] * w[13] + w[14] * w[14] + w[15] * w[15]);
  uint16_t nn[3];
  for (int k = 0; k < 3; ++k) nn[k] = q16(clampd(M16 * 0.5 * (w[13 + k] / nl + 1.0), 0.0, M16));
  memcpy(out + 22, nn, 6);
  uint16_t h = oi_half_bits((float)w[16]);
  memcpy(out + 28, &h, 2);
}

typedef struct {
  const orc_grid* g;
  const orc_filter_params* p;
  const orc_material* mat;
  const int32_t* nodes;
  const float* tris;
  const uint32_t* order;
  const uint32_t* idx;
  const float* normals;
  const float* obj_m2w;
  uint32_t lod;
  uint64_t v0, v1;
  double* wide;
  uint8_t* compact;
  int tid, nthreads;
  const float* uvs;      /* per vertex, 2 each; null: untextured */
  const oi_tex* tex;
  int mtex[4];           /* albedo, glossy, normal, opacity of the material */
  const oi_alpha* alpha; /* null: no opacity map */
} job_t;

/* Symmetric 3x3 eigendecomposition by cyclic Jacobi rotations (Golub and Van
 * Loan, Matrix Computations, section 8.5): each rotation in the plane (p, q)
 * with tan = sign(theta) / (|theta| + sqrt(theta^2 + 1)),
 * theta = (a_qq - a_pp) / (2 a_pq), zeroes a_pq; sweeps stop once the
 * off-diagonal sum of squares is below double rounding of the diagonal's. */
void orc_sym3_eig(const double* S6, double* w, double* V) {
  double a[3][3] = {{S6[0], S6[3], S6[4]}, {S6[3], S6[1], S6[5]}, {S6[4], S6[5], S6[2]}};
  double v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  static const int P[3] = {0, 0, 1}, Q[3] = {1, 2, 2};
  for (int sweep = 0; sweep < 8; ++sweep) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double dg = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (!(off > 4.93e-32 * dg)) break;
    for (int r = 0; r < 3; ++r) {
      const int p = P[r], q = Q[r];
      if (a[p][q] == 0.0) continue;
      const double th = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
      const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
      const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
      for (int k = 0; k < 3; ++k) {
        const double x = a[k][p], y = a[k][q];
        a[k][p] = c * x - sn * y;
        a[k][q] = sn * x + c * y;
      }
      for (int k = 0; k < 3; ++k) {
        const double x = a[p][k], y = a[q][k];
        a[p][k] = c * x - sn * y;
        a[q][k] = sn * x + c * y;
      }
      for (int k = 0; k < 3; ++k) {
        const double x = v[k][p], y = v[k][q];
        v[k][p] = c * x - sn * y;
        v[k][q] = sn * x + c * y;
      }
    }
  }
  int idx[3] = {0, 1, 2};
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2 - i; ++j)
      if (a[idx[j]][idx[j]] < a[idx[j + 1]][idx[j + 1]]) { const int t = idx[j]; idx[j] = idx[j + 1]; idx[j + 1] = t; }
  for (int c = 0; c < 3; ++c) {
    const int src = idx[c];
    w[c] = a[src][src];
    int m = 0;
    for (int k = 1; k < 3; ++k)
      if (fabs(v[k][src]) > fabs(v[m][src])) m = k;
    const double sg = v[m][src] < 0.0 ? -1.0 : 1.0;
    for (int k = 0; k < 3; ++k) V[3 * k + c] = sg * v[k][src];
  }
}

static void filter_voxel(const job_t* J, uint64_t vid, double* w) {
  const orc_grid* g = J->g;
  const orc_filter_params* p = J->p;
  int nx = g->num_voxels[0], ny = g->num_voxels[1], nz = g->num_voxels[2];
  (void)nz;
  int x = (int)(vid % (uint64_t)nx), y = (int)((vid / (uint64_t)nx) % (uint64_t)ny),
      z = (int)(vid / ((uint64_t)nx * (uint64_t)ny));
  float i2w[12];
  oi_m4_to43(oi_m4_mul(m4_from43(g->model_to_world), m4_from43(g->index_to_model)), i2w);
  f3 wlo = F3(g->world_bb_min[0], g->world_bb_min[1], g->world_bb_min[2]);
  f3 whi = F3(g->world_bb_max[0], g->world_bb_max[1], g->world_bb_max[2]);
  f3 ext = sub3(whi, wlo);
  f3 vs = F3(ext.x / (float)nx, ext.y / (float)ny, ext.z / (float)g->num_voxels[2]);
  f3 pm = xpoint(g->index_to_model, F3((float)x + 0.5f, (float)y + 0.5f, (float)z + 0.5f));
  f3 center = xpoint(g->model_to_world, pm);
  float radius = 1.1f * sqrtf(dot3(vs, vs)) / 2.0f;
  float tmaxFixed = vs.x;
  double S[6] = {0, 0, 0, 0, 0, 0}, dif[3] = {0, 0, 0}, spe[3] = {0, 0, 0}, nrm[3] = {0, 0, 0};
  double dist = 0.0, rough = 0.0, ior = 0.0;
  uint32_t hits = 0;
  double* ts = (double*)malloc(sizeof(double) * p->samples_per_voxel);
  const orc_material* m = J->mat;
  for (uint32_t s = 0; s < p->samples_per_voxel; ++s) {
    uint32_t key[2] = {(uint32_t)vid, p->seed};
    uint32_t c0[4] = {s, 0u, J->lod, 0u}, c1[4] = {s, 1u, J->lod, 0u};
    uint32_t r0[4], r1[4];
    orc_philox4x32_10(c0, key, r0);
    orc_philox4x32_10(c1, key, r1);
    f3 oi = add3(F3((float)x, (float)y, (float)z), F3(u01(r0[0]), u01(r0[1]), u01(r0[2])));
    f3 o = xpoint(i2w, oi);
    float zz = 1.0f - 2.0f * u01(r0[3]);
    float rr = sqrtf(fmaxf(0.0f, 1.0f - zz * zz));
    float sn, cs;
    orc_sincos_turns(u01(r1[0]), &sn, &cs);
    f3 d = F3(rr * cs, rr * sn, zz);
    float tmax = p->clip_rays ? sphere_exit(o, d, center, radius) : tmaxFixed;
    hit_t h = oi_trace_alpha(J->nodes, J->tris, o, d, tmax, 0, J->alpha);
    if (h.tri < 0) continue;
    uint32_t prim = J->order[h.tri];
    const uint32_t* tv = &J->idx[3 * (size_t)prim];
    f3 n0 = F3(J->normals[3 * tv[0]], J->normals[3 * tv[0] + 1], J->normals[3 * tv[0] + 2]);
    f3 n1 = F3(J->normals[3 * tv[1]], J->normals[3 * tv[1] + 1], J->normals[3 * tv[1] + 2]);
    f3 n2 = F3(J->normals[3 * tv[2]], J->normals[3 * tv[2] + 1], J->normals[3 * tv[2] + 2]);
    float b0 = (1.0f - h.b1) - h.b2;
    f3 gn = add3(add3(mul3s(n0, b0), mul3s(n1, h.b1)), mul3s(n2, h.b2));
    gn = norm3(gn);
    f3 n = norm3(xvec(J->obj_m2w, gn));
    f3 kd = F3(m->diffuse[0], m->diffuse[1], m->diffuse[2]), ksp = F3(m->specular[0], m->specular[1], m->specular[2]);
    if (J->uvs && (J->mtex[0] >= 0 || J->mtex[1] >= 0 || J->mtex[2] >= 0)) {
      float uv6[6];
      for (int k = 0; k < 3; ++k) {
        uv6[2 * k] = J->uvs[2 * (size_t)tv[k]];
        uv6[2 * k + 1] = J->uvs[2 * (size_t)tv[k] + 1];
      }
      oi_textured_surface(J->tex, J->mtex[0], J->mtex[1], J->mtex[2], uv6, &J->tris[12 * (size_t)h.tri], h.b1, h.b2,
                          &n, &kd, &ksp);
    }
    /* FP64 accumulation of buildS(n, alpha) and the other means */
    double nx_ = n.x, ny_ = n.y, nz_ = n.z, a = m->alpha_x;
    double xx = nx_ * nx_, xy = nx_ * ny_, xz = nx_ * nz_, yy = ny_ * ny_, yz = ny_ * nz_, zq = nz_ * nz_;
    S[0] += xx + a * (yy + zq);
    S[1] += yy + a * (xx + zq);
    S[2] += zq + a * (xx + yy);
    S[3] += xy - a * xy;
    S[4] += xz - a * xz;
    S[5] += yz - a * yz;
    dif[0] += kd.x; dif[1] += kd.y; dif[2] += kd.z;
    spe[0] += ksp.x; spe[1] += ksp.y; spe[2] += ksp.z;
    nrm[0] += nx_;
    nrm[1] += ny_;
    nrm[2] += nz_;
    dist += tmax;
    rough += m->alpha_x;
    ior += m->eta_t;
    ts[hits++] = tmax;
  }
  memset(w, 0, sizeof(double) * 20);
  if (hits == 0) {
    w[16] = 1.0;
    free(ts);
    return;
  }
  double avg = dist / hits;
  double pMesh = (double)hits / (double)p->samples_per_voxel;
  double sig = p->sigma_t;
  double density = -log(1.0 - pMesh) / (avg * sig);
  double nAlpha = (double)p->alpha / sig;
  for (uint32_t it = 0; it < p->estimation_iterations; ++it) {
    double pv;
    if (p->clip_rays) {
      double acc = 0.0;
      for (uint32_t h = 0; h < hits; ++h) acc += exp(-density * sig * ts[h]);
      pv = 1.0 - acc / hits;
    } else {
      pv = 1.0 - exp(-density * sig * (double)tmaxFixed);
    }
    density = density - nAlpha * (pv - pMesh);
  }
  double inv = 1.0 / hits;
  w[0] = density;
  for (int k = 0; k < 6; ++k) w[1 + k] = S[k] * inv;
  if (p->sggx_projection) { /* V diag(max(w, floor * w0)) V^T */
    double ev[3], V[9], l[3];
    orc_sym3_eig(&w[1], ev, V);
    const double lo = (double)p->sggx_floor * (ev[0] > 0.0 ? ev[0] : 0.0);
    for (int k = 0; k < 3; ++k) l[k] = ev[k] > lo ? ev[k] : lo;
    static const int rr[6] = {0, 1, 2, 0, 0, 1}, cc[6] = {0, 1, 2, 1, 2, 2};
    for (int e = 0; e < 6; ++e) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc += l[k] * V[3 * rr[e] + k] * V[3 * cc[e] + k];
      w[1 + e] = acc;
    }
  }
  for (int k = 0; k < 3; ++k) {
    w[7 + k] = dif[k] * inv;
    w[10 + k] = spe[k] * inv;
  }
  const float* w2m = g->world_to_model;
  double mn[3];
  for (int r = 0; r < 3; ++r)
    mn[r] = (double)w2m[r] * nrm[0] * inv + (double)w2m[3 + r] * nrm[1] * inv + (double)w2m[6 + r] * nrm[2] * inv;
  double l = sqrt(mn[0] * mn[0] + mn[1] * mn[1] + mn[2] * mn[2]);
  for (int k = 0; k < 3; ++k) w[13 + k] = mn[k] / l;
  w[16] = ior * inv;
  w[17] = hits;
  w[18] = avg;
  w[19] = rough * inv;
  free(ts);
}

static void* filter_worker(void* arg) {
  job_t* J = (job_t*)arg;
  for (uint64_t v = J->v0 + (uint64_t)J->tid; v < J->v1; v += (uint64_t)J->nthreads) {
    double w[20];
    filter_voxel(J, v, w);
    if (J->wide) memcpy(&J->wide[(v - J->v0) * 20], w, sizeof(w));
    if (J->compact) orc_encode(w, &J->compact[(v - J->v0) * 32]);
  }
  return NULL;
}

int orc_filter(const float* positions, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float* normals,
               const orc_material* mat, const float* obj_m2w, const orc_grid* g, const orc_filter_params* p,
               uint32_t lod, uint64_t v0, uint64_t v1, double* wide_out, uint8_t* compact_out, int threads) {
  return orc_filter_tex(positions, nverts, idx, ntris, normals, NULL, mat, NULL, NULL, NULL, NULL, obj_m2w, g, p, lod,
                        v0, v1, wide_out, compact_out, threads);
}

int orc_filter_tex(const float* positions, uint32_t nverts, const uint32_t* idx, uint32_t ntris, const float* normals,
                   const float* uvs, const orc_material* mat, const orc_texture* albedo, const orc_texture* specular,
                   const orc_texture* normal, const orc_texture* alpha, const float* obj_m2w, const orc_grid* g,
                   const orc_filter_params* p, uint32_t lod, uint64_t v0, uint64_t v1, double* wide_out,
                   uint8_t* compact_out, int threads) {
  if (p->samples_per_voxel == 0 || p->samples_per_voxel > 1024) return -1;
  float* wpos = (float*)malloc(sizeof(float) * 3 * (size_t)nverts);
  for (uint32_t v = 0; v < nverts; ++v) {
    f3 q = xpoint(obj_m2w, F3(positions[3 * v], positions[3 * v + 1], positions[3 * v + 2]));
    wpos[3 * v] = q.x; wpos[3 * v + 1] = q.y; wpos[3 * v + 2] = q.z;
  }
  size_t nn = ntris > 1 ? (size_t)ntris - 1 : 1;
  int32_t* nodes = (int32_t*)malloc(64 * nn);
  uint32_t* order = (uint32_t*)malloc(4 * (size_t)ntris);
  float* tris = (float*)malloc(48 * (size_t)ntris);
  int height = orc_build_bvh_filter(wpos, nverts, idx, ntris, nodes, order, tris);
  if (height < 0 || height > BVH_STACK) {
    free(wpos); free(nodes); free(order); free(tris);
    return -2;
  }
  /* texture maps (unused without texture coordinates) and the opacity map per BVH-order triangle */
  oi_tex tex[4];
  int ntex = 0, mtex[4] = {-1, -1, -1, -1};
  if (uvs) oi_material_maps(mat, albedo, specular, normal, alpha, tex, &ntex, mtex);
  oi_alpha al;
  int* triAlpha = NULL;
  float* triUV = NULL;
  if (mtex[3] >= 0) {
    triAlpha = (int*)malloc(sizeof(int) * (size_t)ntris);
    triUV = (float*)malloc(sizeof(float) * 6 * (size_t)ntris);
    for (uint32_t i = 0; i < ntris; ++i) {
      const uint32_t prim = order[i];
      triAlpha[i] = mtex[3];
      for (int k = 0; k < 3; ++k) {
        triUV[6 * (size_t)i + 2 * k] = uvs[2 * (size_t)idx[3 * (size_t)prim + k]];
        triUV[6 * (size_t)i + 2 * k + 1] = uvs[2 * (size_t)idx[3 * (size_t)prim + k] + 1];
      }
    }
    al.alpha_tex = triAlpha;
    al.uv = triUV;
    al.tex = tex;
  }
  if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (threads < 1) threads = 1;
  job_t* jobs = (job_t*)malloc(sizeof(job_t) * (size_t)threads);
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
  for (int t = 0; t < threads; ++t) {
    job_t J = {g, p, mat, nodes, tris, order, idx, normals, obj_m2w, lod, v0, v1, wide_out, compact_out, t, threads,
               ntex ? uvs : NULL, tex, {mtex[0], mtex[1], mtex[2], mtex[3]}, triAlpha ? &al : NULL};
    jobs[t] = J;
    pthread_create(&th[t], NULL, filter_worker, &jobs[t]);
  }
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  free(jobs); free(th); free(wpos); free(nodes); free(order); free(tris);
  free(triAlpha); free(triUV);
  for (int k = 0; k < ntex; ++k) free(tex[k].texels);
  return height;
}

/* Unit hook for the golden-vector tests: buildS in FP64 as accumulated by the
 * filter oracle (xx yy zz xy xz yz). */
void orc_t_build_s(const float* n, float sigma, double* out) {
  double x = n[0], y = n[1], z = n[2], a = sigma;
  double xx = x * x, xy = x * y, xz = x * z, yy = y * y, yz = y * z, zz = z * z;
  out[0] = xx + a * (yy + zz);
  out[1] = yy + a * (xx + zz);
  out[2] = zz + a * (xx + yy);
  out[3] = xy - a * xy;
  out[4] = xz - a * xz;
  out[5] = yz - a * yz;
}
