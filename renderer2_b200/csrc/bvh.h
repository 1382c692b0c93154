// Triangle BVH that replaces the reference's OptiX GAS/IAS
// (raytracer/src/mesh/mesh.cu:140-168, raytracer/src/scene/scene.cu:188-256)
// and its optixTrace closest-hit query (include/scene/device_scene_impl.hpp:12-31).
//
// Layout in HBM (all arrays 16-byte aligned, read with 128-bit loads):
//   nodes[n-1]  BvhNode, 64 B each: both children's boxes live in the parent so
//               one 64-byte fetch decides which children a ray enters.
//   tris[3n]    float4 per vertex in BVH (Morton) order: v0.xyz|w=orig index,
//               v1.xyz|w=0, v2.xyz|w=0 — the watertight test needs raw vertices.
// Child encoding: c >= 0 is an internal node; c < 0 is a leaf reference
// ~(first | count << 26) (see bvh_leaf_ref).  ch.z holds the node's parent and
// ch.w its depth (build bookkeeping; traversal ignores them).
#pragma once
#include "r2_core.h"
#include "texture.h"

namespace r2 {

struct __align__(16) BvhNode {
  float4 b0;  // child0 lo.x hi.x lo.y hi.y
  float4 b1;  // child1 lo.x hi.x lo.y hi.y
  float4 bz;  // child0 lo.z hi.z, child1 lo.z hi.z
  int4 ch;    // child0, child1, parent, depth
};
static_assert(sizeof(BvhNode) == 64, "BvhNode must be 64 bytes");

// Marker for an absent second child (a BVH over a single leaf).
#define R2_BVH_NONE ((int)0x80000000)

// Alpha-tested triangles: the reference's __anyhit__mesh
// (shaders.optix.cu:132-152) ignores a hit where the material's opacity
// texture reads 0 at the hit's texture coordinates (CMaterial::opaque,
// material.hpp:134-141).  Per BVH-order triangle.
struct BvhAlpha {
  const int* alphaTex;    // texture index of the triangle's opacity map, -1: opaque; null: no alpha test
  const float2* uv;       // 3 texture coordinates per triangle
  const float4* texels;
  const TexInfo* texInfo;
};

// A placed bottom-level BVH of a two-level scene (the reference's OptiX
// instance, sceneobject.cu:330-349).  The top-level BVH's leaves reference
// instances (leaf references with count 0); entering one transforms the ray
// into the instance's object space and continues at its root.  A triangle hit
// inside the instance reports the code tri + vdelta, where tri is the
// triangle's position in the global BVH-order array: codes number the
// triangles of every instance consecutively, instance by instance.
struct __align__(16) BvhInstance {
  float4 w2o[3];  // world -> object: rows (3x3 part | translation)
  int root;       // the instance's BLAS root in the global node array
  int vdelta;     // hit code - global triangle index
  int identity;   // 1: object space is world space (no transform)
  int pad;
};

struct BvhView {
  const BvhNode* nodes;
  const float4* tris;  // 3 per triangle, BVH order
  uint32_t ntris;
  BvhAlpha alpha;      // zero: every triangle opaque
  const BvhInstance* inst;  // two-level scenes: the instances (nodes start with the top level), else null
  const BvhNode* top;       // nodes 0 .. ntop-1 staged in shared memory by the caller (kTop traversals)
  int ntop;
};

R2_HD bool alpha_opaque(const BvhAlpha& a, int tri, float b1, float b2) {
#if defined(__CUDA_ARCH__)
  const int k = __ldg(&a.alphaTex[tri]);
  if (k < 0) return true;
  const float2 tc = tex_coord(__ldg(&a.uv[3 * tri]), __ldg(&a.uv[3 * tri + 1]), __ldg(&a.uv[3 * tri + 2]), b1, b2);
#else
  const int k = a.alphaTex[tri];
  if (k < 0) return true;
  const float2 tc = tex_coord(a.uv[3 * tri], a.uv[3 * tri + 1], a.uv[3 * tri + 2], b1, b2);
#endif
  return tex_lookup(a.texels, a.texInfo[k], tc.x, tc.y).x > 0.0f;
}

struct Hit {
  float t;
  float b1, b2;  // barycentric weights of v1 and v2 (OptiX convention)
  int tri;       // BVH-order triangle index, -1 = miss
};

// Per-ray constants of the watertight ray/triangle test (Woop, Benthin, Wald,
// "Watertight Ray/Triangle Intersection", JCGT 2013).
struct RayPre {
  V3 o, d, invd;
  int kx, ky, kz;
  float Sx, Sy, Sz;
};

R2_HD RayPre make_ray_pre(V3 o, V3 d) {
  RayPre r;
  r.o = o;
  r.d = d;
  r.invd = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  V3 ad = vabs(d);
  int kz = (ad.x > ad.y) ? ((ad.x > ad.z) ? 0 : 2) : ((ad.y > ad.z) ? 1 : 2);
  int kx = kz + 1; if (kx == 3) kx = 0;
  int ky = kx + 1; if (ky == 3) ky = 0;
  if (comp(d, kz) < 0.0f) { int t = kx; kx = ky; ky = t; }
  r.kx = kx; r.ky = ky; r.kz = kz;
  float dz = comp(d, kz);
  r.Sx = comp(d, kx) / dz;
  r.Sy = comp(d, ky) / dz;
  r.Sz = 1.0f / dz;
  return r;
}

// Robust slab test (Ize, "Robust BVH Ray Traversal", JCGT 2013): the far
// distance is scaled by 1 + 2*gamma(3) so boxes are never missed by rounding.
R2_HD bool slab(const RayPre& r, float lox, float hix, float loy, float hiy, float loz,
                float hiz, float tmax, float* tentry) {
  float tx0 = (lox - r.o.x) * r.invd.x, tx1 = (hix - r.o.x) * r.invd.x;
  float ty0 = (loy - r.o.y) * r.invd.y, ty1 = (hiy - r.o.y) * r.invd.y;
  float tz0 = (loz - r.o.z) * r.invd.z, tz1 = (hiz - r.o.z) * r.invd.z;
  float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
  float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
  tf = tf * 1.00000024f;  // 1 + 2*gamma(3) rounded up
  *tentry = tn;
  return tn <= tf;
}

// Watertight test.  Accepts 0 < t and (t, code) lexicographically below the
// current best (t, code) so the closest hit is independent of visiting order;
// kAlpha: and only where the triangle is opaque.  tri is the triangle's
// BVH-order index, code the hit code reported (tri itself in one-level BVHs).
template <bool kAlpha = false>
R2_HD bool tri_test(const RayPre& r, V3 p0, V3 p1, V3 p2, int tri, int code, Hit* best,
                    const BvhAlpha* alpha = nullptr) {
  V3 A = p0 - r.o, B = p1 - r.o, C = p2 - r.o;
  float Az0 = comp(A, r.kz), Bz0 = comp(B, r.kz), Cz0 = comp(C, r.kz);
  float Ax = comp(A, r.kx) - r.Sx * Az0, Ay = comp(A, r.ky) - r.Sy * Az0;
  float Bx = comp(B, r.kx) - r.Sx * Bz0, By = comp(B, r.ky) - r.Sy * Bz0;
  float Cx = comp(C, r.kx) - r.Sx * Cz0, Cy = comp(C, r.ky) - r.Sy * Cz0;
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
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  float det = U + V + W;
  if (det == 0.0f) return false;
  float Az = r.Sz * Az0, Bz = r.Sz * Bz0, Cz = r.Sz * Cz0;
  float T = U * Az + V * Bz + W * Cz;
  float rcp = 1.0f / det;
  float t = T * rcp;
  if (!(t > 0.0f)) return false;
  if (t < best->t || (t == best->t && code < best->tri)) {
    const float b1 = V * rcp, b2 = W * rcp;
    if (kAlpha && !alpha_opaque(*alpha, tri, b1, b2)) return false;
    best->t = t;
    best->b1 = b1;
    best->b2 = b2;
    best->tri = code;
    return true;
  }
  return false;
}

#define R2_BVH_STACK 96
#define R2_LEAF_MAX 16

// Leaf reference: ~(first | count << 26); first < 2^26, count <= 31.
R2_HD int bvh_leaf_ref(int first, int count) { return ~(first | (count << 26)); }
R2_HD int bvh_leaf_first(int ref) { return (~ref) & 0x03FFFFFF; }
R2_HD int bvh_leaf_count(int ref) { return ((~ref) >> 26) & 0x1F; }

// A ray's traversal that can stop after any node or leaf and resume later:
// the per-ray constants, the best hit so far, the node to visit next (or
// kTraceDone), a postponed leaf (0: none) and the depth of the caller-held stack.
struct TraceState {
  RayPre r;
  Hit best;
  int cur;
  int leaf;
  int sp;
  int found;
  uint32_t nodes, tris;  // visits counted by the counting instantiation (kCount)
  V3 wo, wd;             // two-level: the world-space ray, restored when an instance is left
  int vdelta;            // two-level: hit code offset of the instance being traversed (0: top level)
};

constexpr int kTraceDone = 0x7FFFFFFF;  // no node left to visit (never a node index)
constexpr int kInstExit = 0x7FFFFFFE;   // stack marker: leave the current instance (never a node index)

// root: the node the query starts at (0: the tree's root; a child reference
// whose subtree holds every triangle the ray can hit, a leaf included).
R2_HD void trace_begin(TraceState& s, V3 o, V3 d, float tmax, int root = 0) {
  s.r = make_ray_pre(o, d);
  s.wo = o;
  s.wd = d;
  s.vdelta = 0;
  s.best.t = tmax;
  s.best.b1 = s.best.b2 = 0.0f;
  s.best.tri = 0x7FFFFFFF;
  s.cur = root < 0 ? kTraceDone : root;
  s.leaf = root < 0 ? root : 0;
  s.sp = 0;
  s.found = 0;
  s.nodes = s.tris = 0;
}

// The object-space origin and direction of a world-space ray.
R2_HD V3 inst_point(const BvhInstance& in, V3 p) {
  return v3(in.w2o[0].x * p.x + in.w2o[0].y * p.y + in.w2o[0].z * p.z + in.w2o[0].w,
            in.w2o[1].x * p.x + in.w2o[1].y * p.y + in.w2o[1].z * p.z + in.w2o[1].w,
            in.w2o[2].x * p.x + in.w2o[2].y * p.y + in.w2o[2].z * p.z + in.w2o[2].w);
}
R2_HD V3 inst_vector(const BvhInstance& in, V3 d) {
  return v3(in.w2o[0].x * d.x + in.w2o[0].y * d.y + in.w2o[0].z * d.z,
            in.w2o[1].x * d.x + in.w2o[1].y * d.y + in.w2o[1].z * d.z,
            in.w2o[2].x * d.x + in.w2o[2].y * d.y + in.w2o[2].z * d.z);
}

// Next stacked child whose entry distance is not beyond the closest hit.
R2_HD int trace_pop(TraceState& s, const int* stack, const float* stackT) {
  while (s.sp > 0) {
    --s.sp;
    if (stackT[s.sp] <= s.best.t) return stack[s.sp];
  }
  return kTraceDone;
}

// True when every lane of the warp running this loop holds a postponed leaf.
R2_HD bool trace_all_have_leaf(bool mine) {
#if defined(__CUDA_ARCH__)
  return !__any_sync(__activemask(), !mine);
#else
  return mine;
#endif
}

// Visits about maxVisits nodes and triangles; true when the query has
// finished (closest hit in (0, tmax], kAnyHit: the first hit found) with
// s.best.tri the BVH-order index, -1 on a miss.  Speculative while-while
// traversal (Aila and Laine, "Understanding the Efficiency of Ray Traversal on
// GPUs", HPG 2009): inner nodes are visited until every lane of the warp has
// met a leaf, which is postponed while traversal continues; then the lanes
// test their leaves together.  Stack entries hold child references with their
// entry distance.  The builder bounds the tree depth by R2_BVH_STACK so the
// stack cannot overflow.  The closest hit does not depend on the visiting
// order (ties go to the lower triangle index).
//
// kInst (two-level BVHs): a top-level leaf with count 0 is an instance.
// Entering it pushes the node to resume at (without its entry distance) and
// the kInstExit marker, transforms the ray and continues at the instance's
// root; popping the marker restores the world-space ray, after any postponed
// leaf of the instance has been tested.  The stack then holds the top-level
// path, the marker and the instance's path: the builder bounds the sum of the
// two heights plus two by R2_BVH_STACK.
template <bool kAnyHit, bool kCount = false, bool kAlpha = false, bool kInst = false, bool kTop = false>
R2_HD bool trace_advance(const BvhView& bvh, TraceState& s, int* stack, float* stackT, int maxVisits) {
  int budget = maxVisits;
  while (budget > 0) {
    // inner nodes, the first leaf met postponed
    while (s.cur >= 0 && s.cur != kTraceDone && budget > 0) {
      if (kInst && s.cur == kInstExit) {
        if (s.leaf != 0) break;  // the instance's postponed leaf first
        s.r = make_ray_pre(s.wo, s.wd);
        s.vdelta = 0;
        s.cur = trace_pop(s, stack, stackT);
        if (s.cur < 0 && s.leaf == 0) {
          s.leaf = s.cur;
          s.cur = trace_pop(s, stack, stackT);
        }
        if (trace_all_have_leaf(s.leaf != 0)) break;
        continue;
      }
      --budget;
      if (kCount) ++s.nodes;
      const int cur = s.cur;
#if defined(__CUDA_ARCH__)
      float4 b0, b1, bz;
      int4 ch;
      if (kTop && cur < bvh.ntop) {
        b0 = bvh.top[cur].b0;
        b1 = bvh.top[cur].b1;
        bz = bvh.top[cur].bz;
        ch = bvh.top[cur].ch;
      } else {
        b0 = __ldg(&bvh.nodes[cur].b0);
        b1 = __ldg(&bvh.nodes[cur].b1);
        bz = __ldg(&bvh.nodes[cur].bz);
        ch = __ldg(&bvh.nodes[cur].ch);
      }
#else
      const float4 b0 = bvh.nodes[cur].b0;
      const float4 b1 = bvh.nodes[cur].b1;
      const float4 bz = bvh.nodes[cur].bz;
      const int4 ch = bvh.nodes[cur].ch;
#endif
      float t0 = 0.0f, t1 = 0.0f;
      const bool h0 = slab(s.r, b0.x, b0.y, b0.z, b0.w, bz.x, bz.y, s.best.t, &t0);
      const bool h1 = (ch.y != R2_BVH_NONE) && slab(s.r, b1.x, b1.y, b1.z, b1.w, bz.z, bz.w, s.best.t, &t1);
      if (h0 && h1) {
        int nearC = ch.x, farC = ch.y;
        float farT = t1;
        if (t1 < t0) { nearC = ch.y; farC = ch.x; farT = t0; }
        stack[s.sp] = farC;
        stackT[s.sp] = farT;
        ++s.sp;
        s.cur = nearC;
      } else if (h0) {
        s.cur = ch.x;
      } else if (h1) {
        s.cur = ch.y;
      } else {
        s.cur = trace_pop(s, stack, stackT);
      }
      if (s.cur < 0 && s.leaf == 0) {
        s.leaf = s.cur;
        s.cur = trace_pop(s, stack, stackT);
      }
      if (trace_all_have_leaf(s.leaf != 0)) break;
    }
    // postponed leaves, and a leaf met right after one
    while (s.leaf < 0) {
      const int first = bvh_leaf_first(s.leaf);
      const int count = bvh_leaf_count(s.leaf);
      if (kInst && count == 0) {  // enter instance `first`
        --budget;
        s.leaf = 0;
        const BvhInstance& in = bvh.inst[first];
        if (s.cur != kTraceDone) {
          stack[s.sp] = s.cur;
          stackT[s.sp] = -INFINITY;
          ++s.sp;
        }
        stack[s.sp] = kInstExit;
        stackT[s.sp] = -INFINITY;
        ++s.sp;
        if (!in.identity) s.r = make_ray_pre(inst_point(in, s.wo), inst_vector(in, s.wd));
        s.vdelta = in.vdelta;
        s.cur = in.root;
        break;
      }
      budget -= count;
      if (kCount) s.tris += (uint32_t)count;
      for (int i = 0; i < count; ++i) {
        const int tri = first + i;
#if defined(__CUDA_ARCH__)
        const float4 a = __ldg(&bvh.tris[3 * tri + 0]);
        const float4 b = __ldg(&bvh.tris[3 * tri + 1]);
        const float4 c = __ldg(&bvh.tris[3 * tri + 2]);
#else
        const float4 a = bvh.tris[3 * tri + 0];
        const float4 b = bvh.tris[3 * tri + 1];
        const float4 c = bvh.tris[3 * tri + 2];
#endif
        if (tri_test<kAlpha>(s.r, v3(a.x, a.y, a.z), v3(b.x, b.y, b.z), v3(c.x, c.y, c.z), tri,
                             kInst ? tri + s.vdelta : tri, &s.best, &bvh.alpha)) {
          s.found = 1;
          if (kAnyHit) {
            s.leaf = 0;
            s.cur = kTraceDone;
            return true;
          }
        }
      }
      s.leaf = 0;
      if (s.cur < 0) {
        s.leaf = s.cur;
        s.cur = trace_pop(s, stack, stackT);
      }
    }
    if (s.cur == kTraceDone) {
      if (!s.found) s.best.tri = -1;
      return true;
    }
  }
  return false;
}

// The whole query at once; the counting instantiation adds the inner nodes
// visited and the triangles tested to *nodes and *tris.
template <bool kAnyHit, bool kCount = false>
R2_HD Hit bvh_trace(const BvhView& bvh, V3 o, V3 d, float tmax, uint32_t* nodes = nullptr,
                    uint32_t* tris = nullptr, int root = 0) {
  TraceState s;
  trace_begin(s, o, d, tmax, root);
  int stack[R2_BVH_STACK];
  float stackT[R2_BVH_STACK];
  if (bvh.inst) {
    if (bvh.alpha.alphaTex) {
      while (!trace_advance<kAnyHit, kCount, true, true>(bvh, s, stack, stackT, 1 << 30)) {
      }
    } else {
      while (!trace_advance<kAnyHit, kCount, false, true>(bvh, s, stack, stackT, 1 << 30)) {
      }
    }
  } else if (bvh.alpha.alphaTex) {
    while (!trace_advance<kAnyHit, kCount, true>(bvh, s, stack, stackT, 1 << 30)) {
    }
  } else {
    while (!trace_advance<kAnyHit, kCount, false>(bvh, s, stack, stackT, 1 << 30)) {
    }
  }
  if (kCount) {
    *nodes += s.nodes;
    *tris += s.tris;
  }
  return s.best;
}

}  // namespace r2
