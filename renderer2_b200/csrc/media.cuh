// Heterogeneous SGGX media of the path tracer (device + host functions).
//
// Reference: CNVDBMedium (raytracer/include/medium/nvdb_medium_impl.hpp:28-320),
// CMediumInstance (include/medium/medium_instance_impl.hpp:7-45), the SGGX
// microflake phase function (include/medium/sggx_phase_function.hpp:89-233),
// the brick-grid lookups (include/grid_brick/device_grid_brick_impl.hpp:9-33)
// and the medium bounding-box program (src/backend/shaders.optix.cu:192-236).
//
// Grids are the filter's NanoVDB Vec4d grids.  A voxel fetch goes through a
// flat leaf index (one int32 per 8^3 block of the leaves' box) into the
// NanoVDB leaf array: two dependent loads instead of a root/upper/lower walk.
// The brick textures of the reference (indirection, half2 range with 3
// min/max mips, u8 atlas; point sampling, border addressing, normalised
// coordinates) are plain arrays read with the same texel addressing.
// Free-flight distances use log_r2 (identical bits on host and device) in
// place of logf.
#pragma once
#include "shading.h"

namespace r2 {

// A counter-based stream of uniforms: draw i is word i&3 of
// Philox(counter = (sample, bounce, i >> 2, purpose), key = (pixel, seed)).
struct RngStream {
  uint32_t k0, k1, c0, c1, purpose, idx;
  U4 buf;
  R2_HD float next() {
    const uint32_t w = idx & 3u;
    if (w == 0) buf = philox4x32_10(u4(c0, c1, idx >> 2, purpose), k0, k1);
    ++idx;
    return u01(w == 0 ? buf.x : (w == 1 ? buf.y : (w == 2 ? buf.z : buf.w)));
  }
  // The next five draws without consuming them, from the two blocks that hold
  // them (computed together, so lanes of a warp that reach this point compute
  // them at once instead of at different draws); advance() consumes n <= 5.
  R2_HD void peek5(float* u, U4* w0, U4* w1) const {
    const uint32_t b = idx >> 2;
    *w0 = philox4x32_10(u4(c0, c1, b, purpose), k0, k1);
    *w1 = philox4x32_10(u4(c0, c1, b + 1u, purpose), k0, k1);
    for (uint32_t i = 0; i < 5u; ++i) {
      const uint32_t j = (idx & 3u) + i;
      const U4& w = j < 4u ? *w0 : *w1;
      const uint32_t k = j & 3u;
      u[i] = u01(k == 0 ? w.x : (k == 1 ? w.y : (k == 2 ? w.z : w.w)));
    }
  }
  R2_HD void advance(uint32_t n, const U4& w0, const U4& w1) {
    const uint32_t b = idx >> 2;
    idx += n;
    buf = (idx >> 2) == b ? w0 : w1;  // next() recomputes when idx reaches a new block
  }
};
R2_HD RngStream rng_stream(uint32_t pixel, uint32_t seed, uint32_t sample, uint32_t bounce, uint32_t purpose) {
  RngStream r;
  r.k0 = pixel;
  r.k1 = seed;
  r.c0 = sample;
  r.c1 = bounce;
  r.purpose = purpose;
  r.idx = 0;
  r.buf = u4(0, 0, 0, 0);
  return r;
}

// Device view of one medium instance (CHostSceneobject of a Medium:
// sceneobject.cu:50-65, CNVDBMedium::init nvdb_medium.cu:130-173).
struct MediumView {
  M43 modelToWorld, worldToModel;
  V3 aabbMin, aabbMax;       // world box: the model box's two corners transformed
  float filterRenderRatio;   // getFilterRenderRatio (sceneobject.cu:108-114)
  M43 indexToModel, modelToIndex;  // unit box <-> model
  M43 unitToScaled;                // indexToScaledIndex * modelToIndex
  M43 scaledToModel;               // indexToModel * scaledIndexToIndex
  int ibbMin[3], size[3];
  V3 sigmaS;
  float sigmaT;         // max over channels of sigma_a + sigma_s
  float invMaxDensity;  // 1 / max density of the grid
  int hg;               // phase function: 0 SGGX (payload S), 1 Henyey-Greenstein with g
  float g;
  // NanoVDB leaves (16544 B each, payloads at byte 160) and the flat index
  const uint8_t* leaves;
  const int32_t* leafIndex;
  int leafOrigin[3], L[3];
  // brick grid
  const uint32_t* indirection;
  const uint32_t* range;
  const uint32_t* mips[3];
  const uint8_t* atlas;
  int nb[3], ad[3];
};

constexpr int kMediumCodeBase = -1000000;  // closest-hit code of medium m: kMediumCodeBase - m
constexpr int kMaxTrackingSteps = 1 << 20; // largest bound of a tracking loop (the path ends when reached)

// ---------------------------------------------------------------- payload decode / interpolation
// SFilteredData (include/filtering/filtered_data.hpp:10-31; decode 63-89;
// interpolation operators 115-151 with functions.hpp:66-68).
struct FData {
  float density;
  float S[6];  // xx yy zz xy xz yz
  V3 diffuse, specular, normal;
  float ior;
};

R2_HD FData fdata_decode(const r2_voxel& c) {
  const float inv16 = 1.0f / 65535.0f, inv8 = 1.0f / 255.0f;
  FData d;
  d.density = c.density;
  const float sx = c.sigma_x * inv16, sy = c.sigma_y * inv16, sz = c.sigma_z * inv16;
  const float rxy = 2.0f * (c.r_xy * inv16) - 1.0f;
  const float rxz = 2.0f * (c.r_xz * inv16) - 1.0f;
  const float ryz = 2.0f * (c.r_yz * inv16) - 1.0f;
  d.S[0] = sx * sx;
  d.S[1] = sy * sy;
  d.S[2] = sz * sz;
  d.S[3] = rxy * sx * sy;
  d.S[4] = rxz * sx * sz;
  d.S[5] = ryz * sy * sz;
  d.diffuse = v3((float)c.diffuse[0], (float)c.diffuse[1], (float)c.diffuse[2]) * inv8;
  d.specular = v3((float)c.specular[0], (float)c.specular[1], (float)c.specular[2]) * inv8;
  d.normal = normalize(v3((float)c.normal[0], (float)c.normal[1], (float)c.normal[2]) * 2.0f * inv16 - v3(1.0f));
  d.ior = f16_bits_to_f32(c.ior);
  return d;
}

// (1 - t) a + t b with the reference's operator* (the normal is n() scaled)
// and operator+ (the normal sum renormalised).
R2_HD FData fdata_lerp(float t, const FData& a, const FData& b) {
  const float u = 1.0f - t;
  FData r;
  r.density = u * a.density + t * b.density;
  for (int k = 0; k < 6; ++k) r.S[k] = u * a.S[k] + t * b.S[k];
  r.diffuse = a.diffuse * u + b.diffuse * t;
  r.specular = a.specular * u + b.specular * t;
  r.normal = normalize(normalize(a.normal) * u + normalize(b.normal) * t);
  r.ior = u * a.ior + t * b.ior;
  return r;
}

// ReadAccessor::getValue: the leaf's stored payload, else the background
// (zeros with ior = 1).
R2_HD r2_voxel medium_voxel(const MediumView& m, int x, int y, int z) {
  const int bx = (x - m.leafOrigin[0]) >> 3, by = (y - m.leafOrigin[1]) >> 3, bz = (z - m.leafOrigin[2]) >> 3;
  if (x >= m.leafOrigin[0] && y >= m.leafOrigin[1] && z >= m.leafOrigin[2] && bx < m.L[0] && by < m.L[1] &&
      bz < m.L[2]) {
    const int li = m.leafIndex[(size_t)bx + (size_t)by * m.L[0] + (size_t)bz * m.L[0] * m.L[1]];
    if (li >= 0) {
      const size_t off = (size_t)li * 16544 + 160 + (size_t)(((x & 7) << 6) | ((y & 7) << 3) | (z & 7)) * 32;
      r2_voxel v;
#if defined(__CUDA_ARCH__)
      const uint4* src = reinterpret_cast<const uint4*>(m.leaves + off);
      const uint4 lo = __ldg(src), hi = __ldg(src + 1);
      memcpy(reinterpret_cast<uint8_t*>(&v), &lo, 16);
      memcpy(reinterpret_cast<uint8_t*>(&v) + 16, &hi, 16);
#else
      memcpy(&v, m.leaves + off, 32);
#endif
      return v;
    }
  }
  r2_voxel bg;
  memset(&bg, 0, sizeof(bg));
  bg.ior = 0x3C00u;
  return bg;
}

// CNVDBMedium::filteredData: trilinear interpolation of 8 payloads at p (unit box).
R2_HD FData medium_filtered(const MediumView& m, V3 p) {
  const V3 ps = v3(p.x * (float)m.size[0] + (float)m.ibbMin[0] - 0.5f, p.y * (float)m.size[1] + (float)m.ibbMin[1] - 0.5f,
                   p.z * (float)m.size[2] + (float)m.ibbMin[2] - 0.5f);
  const int ix = (int)floorf(ps.x), iy = (int)floorf(ps.y), iz = (int)floorf(ps.z);
  const V3 d = v3(ps.x - (float)ix, ps.y - (float)iy, ps.z - (float)iz);
  const FData d00 = fdata_lerp(d.x, fdata_decode(medium_voxel(m, ix, iy, iz)), fdata_decode(medium_voxel(m, ix + 1, iy, iz)));
  const FData d10 =
      fdata_lerp(d.x, fdata_decode(medium_voxel(m, ix, iy + 1, iz)), fdata_decode(medium_voxel(m, ix + 1, iy + 1, iz)));
  const FData d01 =
      fdata_lerp(d.x, fdata_decode(medium_voxel(m, ix, iy, iz + 1)), fdata_decode(medium_voxel(m, ix + 1, iy, iz + 1)));
  const FData d11 = fdata_lerp(d.x, fdata_decode(medium_voxel(m, ix, iy + 1, iz + 1)),
                               fdata_decode(medium_voxel(m, ix + 1, iy + 1, iz + 1)));
  const FData d0 = fdata_lerp(d.y, d00, d10);
  const FData d1 = fdata_lerp(d.y, d01, d11);
  return fdata_lerp(d.z, d0, d1);
}

// Density at p alone: the density term of medium_filtered with the same
// operations (4-byte loads instead of 32-byte payloads).
R2_HD float voxel_density(const MediumView& m, int x, int y, int z) {
  const int bx = (x - m.leafOrigin[0]) >> 3, by = (y - m.leafOrigin[1]) >> 3, bz = (z - m.leafOrigin[2]) >> 3;
  if (x >= m.leafOrigin[0] && y >= m.leafOrigin[1] && z >= m.leafOrigin[2] && bx < m.L[0] && by < m.L[1] &&
      bz < m.L[2]) {
    const int li = m.leafIndex[(size_t)bx + (size_t)by * m.L[0] + (size_t)bz * m.L[0] * m.L[1]];
    if (li >= 0) {
      const size_t off = (size_t)li * 16544 + 160 + (size_t)(((x & 7) << 6) | ((y & 7) << 3) | (z & 7)) * 32;
#if defined(__CUDA_ARCH__)
      return __ldg(reinterpret_cast<const float*>(m.leaves + off));
#else
      float v;
      memcpy(&v, m.leaves + off, 4);
      return v;
#endif
    }
  }
  return 0.0f;
}
R2_HD float medium_density(const MediumView& m, V3 p) {
  const V3 ps = v3(p.x * (float)m.size[0] + (float)m.ibbMin[0] - 0.5f, p.y * (float)m.size[1] + (float)m.ibbMin[1] - 0.5f,
                   p.z * (float)m.size[2] + (float)m.ibbMin[2] - 0.5f);
  const int ix = (int)floorf(ps.x), iy = (int)floorf(ps.y), iz = (int)floorf(ps.z);
  const float dx = ps.x - (float)ix, dy = ps.y - (float)iy, dz = ps.z - (float)iz;
  const float ux = 1.0f - dx, uy = 1.0f - dy, uz = 1.0f - dz;
  const float d00 = ux * voxel_density(m, ix, iy, iz) + dx * voxel_density(m, ix + 1, iy, iz);
  const float d10 = ux * voxel_density(m, ix, iy + 1, iz) + dx * voxel_density(m, ix + 1, iy + 1, iz);
  const float d01 = ux * voxel_density(m, ix, iy, iz + 1) + dx * voxel_density(m, ix + 1, iy, iz + 1);
  const float d11 = ux * voxel_density(m, ix, iy + 1, iz + 1) + dx * voxel_density(m, ix + 1, iy + 1, iz + 1);
  const float d0 = uy * d00 + dy * d10;
  const float d1 = uy * d01 + dy * d11;
  return uz * d0 + dz * d1;
}

// ---------------------------------------------------------------- rays (ray.hpp:41-91)
struct Ray {
  V3 o, d;
  float tmax;
};
R2_HD Ray make_ray(V3 o, V3 d, float tmax) {
  Ray r;
  r.o = o;
  r.d = d;
  r.tmax = tmax;
  return r;
}
// CRay::transform: the direction is renormalised.
R2_HD Ray ray_transform(const Ray& r, const M43& M) {
  const V3 o = xform_point(M, r.o);
  const V3 e = xform_point(M, r.o + r.d * r.tmax);
  return make_ray(o, normalize(xform_vector(M, r.d)), length(e - o));
}
// CRay::transform2: the direction keeps its length, tmax is in its units.
R2_HD Ray ray_transform2(const Ray& r, const M43& M) {
  const V3 o = xform_point(M, r.o);
  const V3 e = xform_point(M, r.o + r.d * r.tmax);
  const V3 d = xform_vector(M, r.d);
  return make_ray(o, d, length(e - o) / length(d));
}
// CRay::offsetRayOrigin(dir) of a ray: the origin moves, the end point stays.
R2_HD Ray ray_offset(const Ray& r, V3 dir) {
  const V3 end = r.o + r.d * r.tmax;
  const V3 o = offset_ray_origin(r.o, dir);
  return make_ray(o, r.d, length(end - o));
}

// CRay::spawnRay(p0, p1) (ray.hpp:62-69): the origin offset from p0 towards
// p1, the direction (p1 - p0) / |p1 - offset origin| and that length.
R2_HD Ray spawn_ray(V3 p0, V3 p1) {
  const V3 off = offset_ray_origin(p0, normalize(p1 - p0));
  const float tl = length(p1 - off);
  return make_ray(off, (p1 - p0) / tl, tl);
}

// __intersection__volume: nanovdb::Ray::intersects against the world box
// (t0 = 0, t1 = 1e12), reporting the exit when the origin is strictly inside
// and the entry otherwise.  Returns -1 when there is no report.
R2_HD float medium_box_hit(const MediumView& m, V3 o, V3 d) {
  float t0 = 0.0f, t1 = kDefaultTmax;
  const V3 inv = v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  for (int i = 0; i < 3; ++i) {
    float a = comp(m.aabbMin, i), b = comp(m.aabbMax, i);
    if (a >= b) return -1.0f;
    a = (a - comp(o, i)) * comp(inv, i);
    b = (b - comp(o, i)) * comp(inv, i);
    if (a > b) {
      const float t = a;
      a = b;
      b = t;
    }
    if (a > t0) t0 = a;
    if (b < t1) t1 = b;
    if (t0 > t1) return -1.0f;
  }
  if (!(t1 < kDefaultTmax)) return -1.0f;
  const bool inside = o.x > m.aabbMin.x && o.y > m.aabbMin.y && o.z > m.aabbMin.z && o.x < m.aabbMax.x &&
                      o.y < m.aabbMax.y && o.z < m.aabbMax.z;
  return inside ? t1 : t0;
}

// ---------------------------------------------------------------- brick grid (device_grid_brick_impl.hpp)
R2_HD uint32_t brick_word(const uint32_t* a, int nx, int ny, int nz, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return 0u;  // border texel
#if defined(__CUDA_ARCH__)
  return __ldg(&a[(size_t)x + (size_t)y * nx + (size_t)z * nx * ny]);
#else
  return a[(size_t)x + (size_t)y * nx + (size_t)z * nx * ny];
#endif
}
// lookupMajorant: range texel of the brick at mip level `mip` (.y = max).
R2_HD float brick_majorant(const MediumView& m, V3 ipos, int mip) {
  const int bx = (int)floorf(ipos.x) >> 3, by = (int)floorf(ipos.y) >> 3, bz = (int)floorf(ipos.z) >> 3;
  uint32_t w;
  if (mip <= 0) {
    w = brick_word(m.range, m.nb[0], m.nb[1], m.nb[2], bx, by, bz);
  } else {
    w = brick_word(m.mips[mip - 1], m.nb[0] >> mip, m.nb[1] >> mip, m.nb[2] >> mip, bx >> mip, by >> mip, bz >> mip);
  }
  return f16_bits_to_f32((uint16_t)(w >> 16));
}
// lookupDensityBrick: u8 atlas texel decoded with the brick's range.
R2_HD float brick_density(const MediumView& m, V3 ipos) {
  const int ix = (int)floorf(ipos.x), iy = (int)floorf(ipos.y), iz = (int)floorf(ipos.z);
  const int bx = ix >> 3, by = iy >> 3, bz = iz >> 3;
  const uint32_t ptr = brick_word(m.indirection, m.nb[0], m.nb[1], m.nb[2], bx, by, bz);
  const uint32_t rw = brick_word(m.range, m.nb[0], m.nb[1], m.nb[2], bx, by, bz);
  const int ax = (int)((ptr >> 22) & 1023u) * 8 + (ix & 7);
  const int ay = (int)((ptr >> 12) & 1023u) * 8 + (iy & 7);
  const int az = (int)((ptr >> 2) & 1023u) * 8 + (iz & 7);
  uint8_t v = 0;
  if (ax < m.ad[0] && ay < m.ad[1] && az < m.ad[2]) {
    const size_t ai = (size_t)ax + (size_t)ay * m.ad[0] + (size_t)az * m.ad[0] * m.ad[1];
#if defined(__CUDA_ARCH__)
    v = __ldg(&m.atlas[ai]);
#else
    v = m.atlas[ai];
#endif
  }
  const float lo = f16_bits_to_f32((uint16_t)(rw & 0xFFFFu)), hi = f16_bits_to_f32((uint16_t)(rw >> 16));
  return lo + (float)v * (1.0f / 255.0f) * (hi - lo);
}
// CNVDBMedium::stepDDA: distance to the exit of the (8 << mip)^3 cell.
R2_HD float step_dda(V3 pos, V3 invDir, int mip) {
  const float dim = (float)(8 << mip);
  const float ox = invDir.x >= 0.0f ? dim + 0.5f : -0.5f;
  const float oy = invDir.y >= 0.0f ? dim + 0.5f : -0.5f;
  const float oz = invDir.z >= 0.0f ? dim + 0.5f : -0.5f;
  const float tx = (floorf(pos.x * (1.0f / dim)) * dim + ox - pos.x) * invDir.x;
  const float ty = (floorf(pos.y * (1.0f / dim)) * dim + oy - pos.y) * invDir.y;
  const float tz = (floorf(pos.z * (1.0f / dim)) * dim + oz - pos.z) * invDir.z;
  return fminf(tx, fminf(ty, tz));
}

// A collision inside a medium: position, normal, SGGX matrix and ior.
struct MediumEvent {
  int hit;
  V3 pos, normal;
  float S[6];
  float ior;
};

// (diffuse (1 - F) + specular F) sigma_s / sigma_t with F = Fresnel(1, ior).
R2_HD V3 scatter_albedo(const MediumView& m, const FData& fd, V3 dirModel) {
  const V3 n = normalize(fd.normal);
  const float w = fresnel_dielectric(1.0f, fd.ior, fabsf(dot(normalize(-dirModel), n)));
  const V3 a = fd.diffuse * (1.0f - w) + fd.specular * w;
  return v3(a.x * m.sigmaS.x / m.sigmaT, a.y * m.sigmaS.y / m.sigmaT, a.z * m.sigmaS.z / m.sigmaT);
}

R2_HD void fill_event(MediumEvent* ev, const Ray& w, const FData& fd) {
  ev->hit = 1;
  ev->pos = w.o + w.d * w.tmax;
  ev->normal = normalize(fd.normal);
  for (int k = 0; k < 6; ++k) ev->S[k] = fd.S[k];
  ev->ior = fd.ior;
}

R2_HD float inv_majorant(const MediumView& m) { return 1.0f / (m.filterRenderRatio / m.invMaxDensity); }

// CNVDBMedium::sampleInternal (delta tracking against the global majorant),
// model-space ray; *err is set when `limit` steps are reached.
R2_HD V3 medium_sample_internal(const MediumView& m, const Ray& rayModel, RngStream& rng, MediumEvent* ev, int* err,
                                int limit) {
  Ray ray = ray_transform2(rayModel, m.modelToIndex);
  const float invMax = inv_majorant(m);
  if (!(invMax < INFINITY)) return v3(1.0f);  // empty grid: no collision possible
  float t = 0.0f;
  for (int it = 0; it < limit; ++it) {
    t -= log_r2(1.0f - rng.next()) * invMax / m.sigmaT;
    if (t >= ray.tmax) return v3(1.0f);
    const V3 pt = ray.o + ray.d * t;
    if (m.filterRenderRatio * medium_density(m, pt) * invMax > rng.next()) {
      const FData fd = medium_filtered(m, pt);
      ray.tmax = t;
      const Ray w = ray_transform2(ray, m.indexToModel);
      fill_event(ev, w, fd);
      return scatter_albedo(m, fd, w.d);
    }
  }
  *err = 1;
  return v3(0.0f);
}

// CNVDBMedium::sampleDDA (brick-grid majorants; mip starts at 3, +0.25 per
// step, -2 after a tentative collision).
R2_HD V3 medium_sample_dda(const MediumView& m, const Ray& rayModel, RngStream& rng, MediumEvent* ev, int* err,
                           int limit) {
  Ray iray = ray_transform2(rayModel, m.unitToScaled);
  const V3 ri = v3(1.0f / iray.d.x, 1.0f / iray.d.y, 1.0f / iray.d.z);
  float t = 0.0f;
  float tau = -log_r2(1.0f - rng.next());
  float mip = 3.0f;
  for (int it = 0; it < limit; ++it) {
    if (!(t < iray.tmax)) return v3(1.0f);
    const V3 curr = iray.o + iray.d * t;
    const int mi = (int)roundf(mip);
    const float majorant = m.filterRenderRatio * brick_majorant(m, curr, mi);
    const float dt = step_dda(curr, ri, mi);
    const float prevT = t;
    t += dt / m.sigmaT;
    if (t == prevT) return v3(1.0f);
    tau -= majorant * dt;
    mip = fminf(mip + 0.25f, 3.0f);
    if (tau > 0.0f) continue;
    t += tau / (majorant * m.sigmaT);
    if (t >= iray.tmax) return v3(1.0f);
    const float jx = rng.next();
    const float jy = rng.next();
    const float jz = rng.next();
    const float d = brick_density(m, iray.o + iray.d * t + v3(jx, jy, jz) - v3(0.5f));
    if (rng.next() * majorant < d * m.filterRenderRatio) {
      iray.tmax = t;
      const V3 ip = iray.o + iray.d * t;
      const V3 pos = v3((ip.x - (float)m.ibbMin[0]) / (float)m.size[0], (ip.y - (float)m.ibbMin[1]) / (float)m.size[1],
                        (ip.z - (float)m.ibbMin[2]) / (float)m.size[2]);
      const FData fd = medium_filtered(m, pos);
      const Ray w = ray_transform2(iray, m.scaledToModel);
      fill_event(ev, w, fd);
      return scatter_albedo(m, fd, w.d);
    }
    tau = -log_r2(1.0f - rng.next());
    mip = fmaxf(0.0f, mip - 2.0f);
  }
  *err = 1;
  return v3(0.0f);
}

// CNVDBMedium::trInternal (ratio tracking with Russian roulette).
R2_HD float medium_tr_internal(const MediumView& m, const Ray& rayModel, RngStream& rng, int* err, int limit) {
  const Ray ray = ray_transform2(rayModel, m.modelToIndex);
  const float invMax = inv_majorant(m);
  if (!(invMax < INFINITY)) return 1.0f;
  float tr = 1.0f, t = 0.0f;
  for (int it = 0; it < limit; ++it) {
    t -= log_r2(1.0f - rng.next()) * invMax / m.sigmaT;
    if (t >= ray.tmax) return tr;
    const float d = medium_density(m, ray.o + ray.d * t);
    tr *= 1.0f - fmaxf(0.0f, m.filterRenderRatio * d * invMax);
    if (tr < 1.0f) {
      const float p = 1.0f - tr;
      if (rng.next() < p) return 0.0f;
      tr /= 1.0f - p;
    }
  }
  *err = 1;
  return 0.0f;
}

// CNVDBMedium::trDDA.
R2_HD float medium_tr_dda(const MediumView& m, const Ray& rayModel, RngStream& rng, int* err, int limit) {
  const Ray iray = ray_transform2(rayModel, m.unitToScaled);
  const V3 ri = v3(1.0f / iray.d.x, 1.0f / iray.d.y, 1.0f / iray.d.z);
  float tr = 1.0f, t = 0.0f;
  const float volMajorant = 1.0f / inv_majorant(m);
  float tau = -log_r2(1.0f - rng.next());
  float mip = 3.0f;
  for (int it = 0; it < limit; ++it) {
    if (!(t < iray.tmax)) return tr;
    const V3 curr = iray.o + iray.d * t;
    const int mi = (int)roundf(mip);
    const float majorant = m.filterRenderRatio * brick_majorant(m, curr, mi);
    const float dt = step_dda(curr, ri, mi);
    const float prevT = t;
    t += dt / m.sigmaT;
    if (t == prevT) return tr;
    tau -= majorant * dt;
    mip = fminf(mip + 0.25f, 3.0f);
    if (tau > 0.0f) continue;
    t += tau / (majorant * m.sigmaT);
    if (t >= iray.tmax) return tr;
    const float jx = rng.next();
    const float jy = rng.next();
    const float jz = rng.next();
    const float d = brick_density(m, iray.o + iray.d * t + v3(jx, jy, jz) - v3(0.5f));
    if (rng.next() * majorant < d * m.filterRenderRatio) {
      tr *= fmaxf(0.0f, 1.0f - volMajorant / majorant);
      if (tr < 0.1f) {
        const float prob = 1.0f - tr;
        if (rng.next() < prob) return 0.0f;
        tr /= 1.0f - prob;
      }
    }
    tau = -log_r2(1.0f - rng.next());
    mip = fmaxf(0.0f, mip - 2.0f);
  }
  *err = 1;
  return 0.0f;
}

// CMediumInstance::sample: world-space ray; returns the albedo weight (1 when
// the ray passes) and, on a collision, the event in world space.
R2_HD V3 instance_sample(const MediumView& m, const Ray& rayWorld, bool dda, RngStream& rng, MediumEvent* ev, int* err,
                         int limit) {
  const Ray rm = ray_transform2(rayWorld, m.worldToModel);
  ev->hit = 0;
  const V3 a = dda ? medium_sample_dda(m, rm, rng, ev, err, limit) : medium_sample_internal(m, rm, rng, ev, err, limit);
  if (ev->hit) {
    ev->pos = xform_point(m.modelToWorld, ev->pos);
    ev->normal = normalize(xform_vector(m.modelToWorld, ev->normal));
  }
  return a;
}

// CMediumInstance::tr.
R2_HD float instance_tr(const MediumView& m, const Ray& rayWorld, bool dda, RngStream& rng, int* err, int limit) {
  const Ray rm = ray_transform2(rayWorld, m.worldToModel);
  return dda ? medium_tr_dda(m, rm, rng, err, limit) : medium_tr_internal(m, rm, rng, err, limit);
}

// CNVDBMedium::moveToVoxelBorder (model space): the origin moves to just
// before the exit of its voxel.
R2_HD Ray medium_move_to_voxel_border(const MediumView& m, const Ray& rayModel) {
  const Ray ri = ray_transform(rayModel, m.modelToIndex);
  const V3 ibb = v3((float)m.ibbMin[0], (float)m.ibbMin[1], (float)m.ibbMin[2]);
  const V3 sz = v3((float)m.size[0], (float)m.size[1], (float)m.size[2]);
  const V3 ip = v3(ri.o.x * sz.x + ibb.x, ri.o.y * sz.y + ibb.y, ri.o.z * sz.z + ibb.z);
  const V3 vlo = v3((floorf(ip.x) - ibb.x) / sz.x, (floorf(ip.y) - ibb.y) / sz.y, (floorf(ip.z) - ibb.z) / sz.z);
  const V3 vhi = v3((ceilf(ip.x) - ibb.x) / sz.x, (ceilf(ip.y) - ibb.y) / sz.y, (ceilf(ip.z) - ibb.z) / sz.z);
  const float eps = 1.1920928955078125e-07f;  // FLT_EPSILON
  const float gamma = (3.0f * eps) / (1.0f - 3.0f * eps);
  float t1 = ri.tmax;
  for (int i = 0; i < 3; ++i) {
    const float inv = 1.0f / comp(ri.d, i);
    float tn = (comp(vlo, i) - comp(ri.o, i)) * inv;
    float tf = (comp(vhi, i) - comp(ri.o, i)) * inv;
    if (tn > tf) {
      const float tt = tn;
      tn = tf;
      tf = tt;
    }
    tf *= 1.0f + 2.0f * gamma;
    t1 = tf < t1 ? tf : t1;
  }
  t1 *= (1.0f - kRayOffset);
  const Ray moved = make_ray(ri.o + ri.d * t1, ri.d, ri.tmax - t1);
  return ray_offset(ray_transform(moved, m.indexToModel), -rayModel.d);
}
// CMediumInstance::moveToVoxelBorder (world space).
R2_HD Ray instance_move_to_voxel_border(const MediumView& m, const Ray& rayWorld) {
  const Ray rm = ray_transform(rayWorld, m.worldToModel);
  const Ray moved = medium_move_to_voxel_border(m, rm);
  return ray_offset(ray_transform(moved, m.modelToWorld), -rayWorld.d);
}

// ---------------------------------------------------------------- SGGX microflake phase function
struct Sggx {
  float S[6];    // xx yy zz xy xz yz
  float inv[9];  // glm::inverse(S), column major
  V3 normal;
};

R2_HD float s_at(const float* S, int r, int c) {
  if (r == c) return S[r];
  const int a = r < c ? r : c, b = r < c ? c : r;
  return (a == 0 && b == 1) ? S[3] : ((a == 0) ? S[4] : S[5]);
}
// Determinant of a symmetric 3x3 by cofactors of the first column.
R2_HD float det3(const float* S) {
  return s_at(S, 0, 0) * (s_at(S, 1, 1) * s_at(S, 2, 2) - s_at(S, 2, 1) * s_at(S, 1, 2)) -
         s_at(S, 1, 0) * (s_at(S, 0, 1) * s_at(S, 2, 2) - s_at(S, 2, 1) * s_at(S, 0, 2)) +
         s_at(S, 2, 0) * (s_at(S, 0, 1) * s_at(S, 1, 2) - s_at(S, 1, 1) * s_at(S, 0, 2));
}
// Inverse through the adjugate divided by the determinant.
R2_HD void mat3_inverse(const float* S, float* inv) {
  float m[3][3];  // m[col][row]
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) m[c][r] = s_at(S, r, c);
  const float o = 1.0f / (m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) -
                          m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
                          m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]));
  inv[0] = +(m[1][1] * m[2][2] - m[2][1] * m[1][2]) * o;
  inv[3] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * o;
  inv[6] = +(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * o;
  inv[1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * o;
  inv[4] = +(m[0][0] * m[2][2] - m[2][0] * m[0][2]) * o;
  inv[7] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * o;
  inv[2] = +(m[0][1] * m[1][2] - m[1][1] * m[0][2]) * o;
  inv[5] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * o;
  inv[8] = +(m[0][0] * m[1][1] - m[1][0] * m[0][1]) * o;
}
R2_HD V3 smul(const float* S, V3 w) {
  return v3(s_at(S, 0, 0) * w.x + s_at(S, 1, 0) * w.y + s_at(S, 2, 0) * w.z,
            s_at(S, 0, 1) * w.x + s_at(S, 1, 1) * w.y + s_at(S, 2, 1) * w.z,
            s_at(S, 0, 2) * w.x + s_at(S, 1, 2) * w.y + s_at(S, 2, 2) * w.z);
}
R2_HD Sggx make_sggx(const float* S, V3 normal) {
  Sggx g;
  for (int k = 0; k < 6; ++k) g.S[k] = S[k];
  mat3_inverse(S, g.inv);
  g.normal = normal;
  return g;
}
// D(w) = 1 / (pi sqrt|det S| (w^T S^-1 w)^2), the product with M_PI in double.
R2_HD float sggx_D(const Sggx& g, V3 w) {
  const V3 iw = v3(g.inv[0] * w.x + g.inv[3] * w.y + g.inv[6] * w.z, g.inv[1] * w.x + g.inv[4] * w.y + g.inv[7] * w.z,
                   g.inv[2] * w.x + g.inv[5] * w.y + g.inv[8] * w.z);
  const float v = dot(w, iw);
  return (float)(1.0 / (kPiD * (double)sqrtf(fabsf(det3(g.S))) * (double)v * (double)v));
}
R2_HD float sggx_sigma(const Sggx& g, V3 w) { return sqrtf(fmaxf(dot(w, smul(g.S, w)), 0.0f)); }

// CCoordinateFrame::fromNormal2 (objects.hpp:42-58, Frisvad's basis).
R2_HD void frame_frisvad(V3 N, V3* T, V3* B) {
  if (N.z < -0.9999999f) {
    *T = v3(0.0f, -1.0f, 0.0f);
    *B = v3(-1.0f, 0.0f, 0.0f);
  } else {
    const float a = 1.0f / (1.0f + N.z);
    const float b = -N.x * N.y * a;
    *T = normalize(v3(1.0f - N.x * N.x * a, b, -N.x));
    *B = normalize(v3(b, 1.0f - N.y * N.y * a, -N.y));
  }
}

// CSGGXMicroflakeDistribution::sampleVNDF (sggx_phase_function.hpp:116-145):
// visible normals of the direction `normal` (the reference ignores w_i).
R2_HD V3 sggx_sample_vndf(const Sggx& g, float u1, float u2) {
  V3 T, B;
  frame_frisvad(g.normal, &T, &B);
  const V3 wk = B, wj = T, wi = g.normal;
  const float Skk = dot(wk, smul(g.S, wk)), Skj = dot(wk, smul(g.S, wj)), Ski = dot(wk, smul(g.S, wi));
  const float Sjj = dot(wj, smul(g.S, wj)), Sji = dot(wj, smul(g.S, wi)), Sii = dot(wi, smul(g.S, wi));
  const float P[6] = {Skk, Sjj, Sii, Skj, Ski, Sji};
  const float temp = sqrtf(Sjj * Sii - Sji * Sji);
  const V3 Mk = v3(sqrtf(fabsf(det3(P))) / temp, 0.0f, 0.0f);
  const float scaling = 1.0f / sqrtf(Sii);
  const V3 Mj = v3(-(Ski * Sji - Skj * Sii) / temp, temp, 0.0f) * scaling;
  const V3 Mi = v3(Ski, Sji, Sii) * scaling;
  const float sq = sqrtf(u1);
  float sn, cs;
  sincos_turns(u2, &sn, &cs);
  const float u = sq * cs, v = sq * sn;
  const float w = sqrtf(1.0f - u * u - v * v);
  const V3 wm = normalize(Mk * u + Mj * v + Mi * w);
  return normalize(wk * wm.x + wj * wm.y + wi * wm.z);
}
R2_HD float sggx_p_specular(const Sggx& g, V3 wo, V3 wi) {
  const V3 wh = normalize(wi + wo);
  return sggx_D(g, wh) / (4.0f * sggx_sigma(g, wo));
}
// CSGGXPhaseFunction::p: the diffuse lobe draws a visible normal (2 uniforms).
R2_HD float sggx_p(const Sggx& g, float ior, V3 wo, V3 wi, RngStream& rng) {
  const float w = fresnel_dielectric(1.0f, ior, fabsf(dot(normalize(wo), g.normal)));
  const float a = rng.next();
  const float b = rng.next();
  const V3 wm = sggx_sample_vndf(g, a, b);
  const float pd = (float)((double)fmaxf(dot(wi, wm), 0.0f) / kPiD);
  return pd * (1.0f - w) + sggx_p_specular(g, wo, wi) * w;
}
// CSGGXPhaseFunction::sampleP: specular with probability F, else the diffuse
// lobe (visible normal, then a cosine direction around it).
R2_HD float sggx_sample_p(const Sggx& g, float ior, V3 wo, V3* wi, RngStream& rng) {
  const float w = fresnel_dielectric(1.0f, ior, fabsf(dot(normalize(wo), g.normal)));
  if (rng.next() < w) {
    const float a = rng.next();
    const float b = rng.next();
    const V3 wm = sggx_sample_vndf(g, a, b);
    *wi = reflect(-wo, wm);
    return sggx_p_specular(g, wo, *wi);
  }
  const float a = rng.next();
  const float b = rng.next();
  const V3 wn = sggx_sample_vndf(g, a, b);
  const Frame fr = frame_from_normal(wn);
  const float c1 = rng.next();
  const float c2 = rng.next();
  *wi = normalize(to_world(fr, cosine_sample_hemisphere(c1, c2)));
  return (float)((double)fmaxf(dot(*wi, wn), 0.0f) / kPiD);
}

// ---------------------------------------------------------------- resumable tracking
// The four tracking loops above, cut into single steps so that a warp can
// interleave many segments of different lengths (a lane whose segment ends
// takes the next one from a queue).  Each step is one loop iteration of the
// corresponding function with the same operations and random draws, so a
// segment tracked step by step gives the same result as the loop.
enum TrackStatus : int { kTrackRunning = 0, kTrackDone = 1, kTrackCollide = 2, kTrackError = 3, kTrackPending = 4 };

struct TrackState {
  V3 o, d, ri;  // ray in the tracking space (unit box, or scaled index box for the DDA), 1/d
  float tmax, t, tau, mip, tr, invMax;
  float maj;    // DDA: the majorant of a tentative collision waiting for its test
  int steps;
  RngStream rng;
};

// Start of sampleInternal / sampleDDA (kSample) or trInternal / trDDA for a
// world-space ray through the instance.
template <bool kDDA, bool kSample>
R2_HD int track_init(const MediumView& m, const Ray& rayWorld, TrackState* s, int limit) {
  const Ray rm = ray_transform2(rayWorld, m.worldToModel);
  s->t = 0.0f;
  s->tr = 1.0f;
  s->steps = kMaxTrackingSteps - limit;  // track_step ends the loop at kMaxTrackingSteps: after `limit` steps
  if (kDDA) {
    const Ray iray = ray_transform2(rm, m.unitToScaled);
    s->o = iray.o;
    s->d = iray.d;
    s->tmax = iray.tmax;
    s->ri = v3(1.0f / iray.d.x, 1.0f / iray.d.y, 1.0f / iray.d.z);
    if (!kSample) s->invMax = 1.0f / inv_majorant(m);  // the volume majorant of trDDA
    s->tau = -log_r2(1.0f - s->rng.next());
    s->mip = 3.0f;
  } else {
    const Ray ray = ray_transform2(rm, m.modelToIndex);
    s->o = ray.o;
    s->d = ray.d;
    s->tmax = ray.tmax;
    s->invMax = inv_majorant(m);
    if (!(s->invMax < INFINITY)) return kTrackDone;
  }
  return kTrackRunning;
}

// The collision at parameter t of the tracking-space ray (o, d) of a sampled
// segment: the event in world space and the albedo weight, as sampleInternal /
// sampleDDA compute them when their test accepts.
template <bool kDDA>
R2_HD V3 track_collision(const MediumView& m, V3 o, V3 d, float t, MediumEvent* ev) {
  FData fd;
  Ray w;
  if (kDDA) {
    const V3 ip = o + d * t;
    const V3 pos = v3((ip.x - (float)m.ibbMin[0]) / (float)m.size[0], (ip.y - (float)m.ibbMin[1]) / (float)m.size[1],
                      (ip.z - (float)m.ibbMin[2]) / (float)m.size[2]);
    fd = medium_filtered(m, pos);
    w = ray_transform2(make_ray(o, d, t), m.scaledToModel);
  } else {
    fd = medium_filtered(m, o + d * t);
    w = ray_transform2(make_ray(o, d, t), m.indexToModel);
  }
  fill_event(ev, w, fd);
  const V3 albedo = scatter_albedo(m, fd, w.d);
  ev->pos = xform_point(m.modelToWorld, ev->pos);
  ev->normal = normalize(xform_vector(m.modelToWorld, ev->normal));
  return albedo;
}

// The DDA iteration in two parts.  track_dda_advance takes one step across
// the brick grid's majorant cells and returns kTrackPending when the optical
// depth runs out inside the segment (a tentative collision at s.t, majorant
// in s.maj); track_dda_collide then tests it against the brick density.  A
// persistent tracker can hold a pending test while the warp's other lanes
// step on, and test all pending collisions together: each lane performs the
// same operations in the same order as track_step.
template <bool kSample>
R2_HD int track_dda_advance(const MediumView& m, TrackState& s) {
  if (s.steps >= kMaxTrackingSteps) return kTrackError;
  ++s.steps;
  if (!(s.t < s.tmax)) return kTrackDone;
  const V3 curr = s.o + s.d * s.t;
  const int mi = (int)roundf(s.mip);
  const float majorant = m.filterRenderRatio * brick_majorant(m, curr, mi);
  const float dt = step_dda(curr, s.ri, mi);
  const float prevT = s.t;
  s.t += dt / m.sigmaT;
  if (s.t == prevT) return kTrackDone;
  s.tau -= majorant * dt;
  s.mip = fminf(s.mip + 0.25f, 3.0f);
  if (s.tau > 0.0f) return kTrackRunning;
  s.t += s.tau / (majorant * m.sigmaT);
  if (s.t >= s.tmax) return kTrackDone;
  s.maj = majorant;
  return kTrackPending;
}

template <bool kSample>
R2_HD int track_dda_collide(const MediumView& m, TrackState& s) {
  const float majorant = s.maj;
  // draws: jitter x, y, z, acceptance, then the roulette (transmittance
  // only, after a real collision that drops tr below 0.1) and the next
  // free-flight sample, in that order
  float u[5];
  U4 w0, w1;
  s.rng.peek5(u, &w0, &w1);
  const float d = brick_density(m, s.o + s.d * s.t + v3(u[0], u[1], u[2]) - v3(0.5f));
  if (u[3] * majorant < d * m.filterRenderRatio) {
    if (kSample) {
      s.rng.advance(4, w0, w1);
      return kTrackCollide;
    }
    s.tr *= fmaxf(0.0f, 1.0f - s.invMax / majorant);
    if (s.tr < 0.1f) {
      const float prob = 1.0f - s.tr;
      s.rng.advance(5, w0, w1);
      if (u[4] < prob) {
        s.tr = 0.0f;
        return kTrackDone;
      }
      s.tr /= 1.0f - prob;
      s.tau = -log_r2(1.0f - s.rng.next());
      s.mip = fmaxf(0.0f, s.mip - 2.0f);
      return kTrackRunning;
    }
  }
  s.rng.advance(5, w0, w1);
  s.tau = -log_r2(1.0f - u[4]);
  s.mip = fmaxf(0.0f, s.mip - 2.0f);
  return kTrackRunning;
}

// One iteration.  kSample: kTrackCollide leaves the collision at s.t (see
// track_collision).  Transmittance: kTrackDone leaves the estimate in s.tr.
template <bool kDDA, bool kSample>
R2_HD int track_step(const MediumView& m, TrackState& s) {
  if (kDDA) {
    const int st = track_dda_advance<kSample>(m, s);
    return st == kTrackPending ? track_dda_collide<kSample>(m, s) : st;
  }
  if (s.steps >= kMaxTrackingSteps) return kTrackError;
  ++s.steps;
  s.t -= log_r2(1.0f - s.rng.next()) * s.invMax / m.sigmaT;
  if (s.t >= s.tmax) return kTrackDone;
  const V3 pt = s.o + s.d * s.t;
  const float dens = medium_density(m, pt);
  if (kSample) return m.filterRenderRatio * dens * s.invMax > s.rng.next() ? kTrackCollide : kTrackRunning;
  s.tr *= 1.0f - fmaxf(0.0f, m.filterRenderRatio * dens * s.invMax);
  if (s.tr < 1.0f) {
    const float p = 1.0f - s.tr;
    if (s.rng.next() < p) {
      s.tr = 0.0f;
      return kTrackDone;
    }
    s.tr /= 1.0f - p;
  }
  return kTrackRunning;
}

// ---------------------------------------------------------------- Henyey-Greenstein
// (include/medium/henyey_greenstein_phase_function.hpp:22-50, coordinateSystem
// and sphericalDirection of include/utility/functions.hpp:29-47); the media of
// scene objects with a "G" key use it instead of the SGGX lobes.
R2_HD float phase_hg(float cosTheta, float g) {
  const float denom = 1.0f + g * g + 2.0f * g * cosTheta;
  return (float)((double)(1.0f - g * g) / (4.0 * kPiD * (double)denom * (double)sqrtf(denom)));
}
R2_HD float hg_sample_p(float g, V3 wo, V3* wi, RngStream& rng) {
  const float u1 = rng.next();
  const float u2 = rng.next();
  float cosTheta;
  if (fabsf(g) < 1e-3f) {
    cosTheta = 1.0f - 2.0f * u1;
  } else {
    const float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
    cosTheta = (1.0f + g * g - sq * sq) / (2.0f * g);
  }
  const float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
  float s, c;
  sincos_turns(u2, &s, &c);  // phi = 2 pi u2
  const V3 v1 = fabsf(wo.x) > fabsf(wo.y) ? v3(-wo.z, 0.0f, wo.x) / sqrtf(wo.x * wo.x + wo.z * wo.z)
                                          : v3(0.0f, wo.z, -wo.y) / sqrtf(wo.y * wo.y + wo.z * wo.z);
  const V3 v2 = cross(wo, v1);
  *wi = v1 * (sinTheta * c) + v2 * (sinTheta * s) + (-wo) * cosTheta;
  return phase_hg(-cosTheta, g);
}

}  // namespace r2
