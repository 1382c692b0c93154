// Seeded synthetic inputs standing in for the reference's thesis assets (the
// Xfrog OBJ trees and HDR maps are not available): displaced icospheres and
// leaf-quad foliage.  Deterministic functions of their parameters.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <map>
#include <utility>
#include <vector>

#include "r2_core.h"
#include "gen.h"

namespace r2 {

namespace {

// Philox-driven uniform doubles in [0, 1) with 53 random bits.
struct Rng {
  uint32_t key0, key1;
  uint32_t ctr = 0;
  U4 buf;
  int left = 0;
  Rng(uint32_t seed, uint32_t stream) : key0(seed), key1(stream ^ 0x5eed1234u) {}
  uint32_t next32() {
    if (left == 0) {
      buf = philox4x32_10(u4(ctr++, 0u, 0u, 0u), key0, key1);
      left = 4;
    }
    uint32_t v = (left == 4) ? buf.x : (left == 3) ? buf.y : (left == 2) ? buf.z : buf.w;
    --left;
    return v;
  }
  double uniform() {
    uint64_t a = next32() >> 5, b = next32() >> 6;
    return (double)(a * 67108864ull + b) * (1.0 / 9007199254740992.0);
  }
  double normal() {
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
  }
};

uint32_t hash3(int x, int y, int z, uint32_t seed) {
  U4 h = philox4x32_10(u4((uint32_t)x, (uint32_t)y, (uint32_t)z, 0x9e37u), seed, 0x7f4a7c15u);
  return h.x;
}

double lattice(int x, int y, int z, uint32_t seed) {
  return (double)hash3(x, y, z, seed) * (2.0 / 4294967295.0) - 1.0;
}

double fade(double t) { return t * t * (3.0 - 2.0 * t); }

}  // namespace

// Value noise: smooth interpolation of hashed lattice values in [-1, 1].
double value_noise(double px, double py, double pz, uint32_t seed) {
  double fx = floor(px), fy = floor(py), fz = floor(pz);
  int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  double tx = fade(px - fx), ty = fade(py - fy), tz = fade(pz - fz);
  double c[2][2][2];
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) c[dz][dy][dx] = lattice(ix + dx, iy + dy, iz + dz, seed);
  double x00 = c[0][0][0] + (c[0][0][1] - c[0][0][0]) * tx;
  double x10 = c[0][1][0] + (c[0][1][1] - c[0][1][0]) * tx;
  double x01 = c[1][0][0] + (c[1][0][1] - c[1][0][0]) * tx;
  double x11 = c[1][1][0] + (c[1][1][1] - c[1][1][0]) * tx;
  double y0 = x00 + (x10 - x00) * ty;
  double y1 = x01 + (x11 - x01) * ty;
  return y0 + (y1 - y0) * tz;
}

void smooth_normals(const std::vector<float>& pos, const std::vector<uint32_t>& idx, std::vector<float>* nrm) {
  size_t nv = pos.size() / 3;
  std::vector<double> acc(3 * nv, 0.0);
  for (size_t t = 0; t < idx.size() / 3; ++t) {
    uint32_t i0 = idx[3 * t], i1 = idx[3 * t + 1], i2 = idx[3 * t + 2];
    double e1[3], e2[3];
    for (int k = 0; k < 3; ++k) {
      e1[k] = (double)pos[3 * i1 + k] - pos[3 * i0 + k];
      e2[k] = (double)pos[3 * i2 + k] - pos[3 * i0 + k];
    }
    double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    for (uint32_t v : {i0, i1, i2})
      for (int k = 0; k < 3; ++k) acc[3 * v + k] += n[k];
  }
  nrm->resize(3 * nv);
  for (size_t v = 0; v < nv; ++v) {
    double l = sqrt(acc[3 * v] * acc[3 * v] + acc[3 * v + 1] * acc[3 * v + 1] + acc[3 * v + 2] * acc[3 * v + 2]);
    if (l == 0.0) l = 1.0;
    for (int k = 0; k < 3; ++k) (*nrm)[3 * v + k] = (float)(acc[3 * v + k] / l);
  }
}

void gen_icosphere(uint32_t subdiv, float amplitude, uint32_t seed, std::vector<float>* pos,
                   std::vector<uint32_t>* idx, std::vector<float>* nrm) {
  const double t = (1.0 + sqrt(5.0)) / 2.0;
  std::vector<double> P = {-1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, 0, 0, -1, t, 0, 1, t,
                           0, -1, -t, 0, 1, -t, t, 0, -1, t, 0, 1, -t, 0, -1, -t, 0, 1};
  std::vector<uint32_t> F = {0, 11, 5, 0, 5, 1,  0, 1, 7,   0, 7,  10, 0, 10, 11, 1, 5, 9, 5, 11,
                             4, 11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9,  4, 3, 4,  2,  3, 2, 6, 3,
                             6, 8,  3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8,  6,  7, 9, 8, 1};
  auto norm = [&](uint32_t v) {
    double l = sqrt(P[3 * v] * P[3 * v] + P[3 * v + 1] * P[3 * v + 1] + P[3 * v + 2] * P[3 * v + 2]);
    for (int k = 0; k < 3; ++k) P[3 * v + k] /= l;
  };
  for (uint32_t v = 0; v < 12; ++v) norm(v);
  for (uint32_t s = 0; s < subdiv; ++s) {
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> mid;
    auto midpoint = [&](uint32_t a, uint32_t b) {
      std::pair<uint32_t, uint32_t> key = a < b ? std::make_pair(a, b) : std::make_pair(b, a);
      auto it = mid.find(key);
      if (it != mid.end()) return it->second;
      uint32_t v = (uint32_t)(P.size() / 3);
      for (int k = 0; k < 3; ++k) P.push_back(0.5 * (P[3 * a + k] + P[3 * b + k]));
      norm(v);
      mid[key] = v;
      return v;
    };
    std::vector<uint32_t> G;
    G.reserve(F.size() * 4);
    for (size_t f = 0; f < F.size() / 3; ++f) {
      uint32_t a = F[3 * f], b = F[3 * f + 1], c = F[3 * f + 2];
      uint32_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
      uint32_t tri[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
      G.insert(G.end(), tri, tri + 12);
    }
    F.swap(G);
  }
  size_t nv = P.size() / 3;
  pos->resize(3 * nv);
  for (size_t v = 0; v < nv; ++v) {
    double x = P[3 * v], y = P[3 * v + 1], z = P[3 * v + 2];
    double r = 1.0 + (double)amplitude * value_noise(4.0 * x, 4.0 * y, 4.0 * z, seed);
    (*pos)[3 * v] = (float)(r * x);
    (*pos)[3 * v + 1] = (float)(r * y);
    (*pos)[3 * v + 2] = (float)(r * z);
  }
  *idx = F;
  smooth_normals(*pos, *idx, nrm);
}

void gen_foliage(uint32_t nQuads, uint32_t nBranches, float clustered, uint32_t seed, std::vector<float>* pos,
                 std::vector<uint32_t>* idx, std::vector<float>* nrm) {
  Rng rng(seed, 1u);
  std::vector<double> ctrl((size_t)nBranches * 12);
  for (auto& c : ctrl) c = 0.1 + 0.8 * rng.uniform();
  pos->clear();
  idx->clear();
  nrm->clear();
  pos->reserve((size_t)nQuads * 12);
  nrm->reserve((size_t)nQuads * 12);
  idx->reserve((size_t)nQuads * 6);
  for (uint32_t q = 0; q < nQuads; ++q) {
    double c[3];
    if (nBranches > 0 && rng.uniform() < clustered) {
      uint32_t b = (uint32_t)(rng.uniform() * nBranches);
      if (b >= nBranches) b = nBranches - 1;
      double u = rng.uniform(), iu = 1.0 - u;
      double w[4] = {iu * iu * iu, 3 * u * iu * iu, 3 * u * u * iu, u * u * u};
      for (int k = 0; k < 3; ++k) {
        double v = 0.0;
        for (int j = 0; j < 4; ++j) v += w[j] * ctrl[(size_t)b * 12 + 3 * j + k];
        c[k] = v + 0.02 * rng.normal();
      }
    } else {
      for (int k = 0; k < 3; ++k) c[k] = rng.uniform();
    }
    for (int k = 0; k < 3; ++k) c[k] = c[k] < 0.0 ? 0.0 : (c[k] > 1.0 ? 1.0 : c[k]);
    // random orientation: normal uniform on the sphere, tangent frame rotated by phi
    double z = 1.0 - 2.0 * rng.uniform(), phi = 2.0 * M_PI * rng.uniform();
    double r = sqrt(fmax(0.0, 1.0 - z * z));
    double n[3] = {r * cos(phi), r * sin(phi), z};
    double a[3] = {fabs(n[0]) > 0.9 ? 0.0 : 1.0, fabs(n[0]) > 0.9 ? 1.0 : 0.0, 0.0};
    double t1[3] = {n[1] * a[2] - n[2] * a[1], n[2] * a[0] - n[0] * a[2], n[0] * a[1] - n[1] * a[0]};
    double l1 = sqrt(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
    for (int k = 0; k < 3; ++k) t1[k] /= l1;
    double t2[3] = {n[1] * t1[2] - n[2] * t1[1], n[2] * t1[0] - n[0] * t1[2], n[0] * t1[1] - n[1] * t1[0]};
    double rot = 2.0 * M_PI * rng.uniform(), cr = cos(rot), sr = sin(rot);
    double u[3], v[3];
    for (int k = 0; k < 3; ++k) {
      u[k] = cr * t1[k] + sr * t2[k];
      v[k] = -sr * t1[k] + cr * t2[k];
    }
    double h = 0.5 * (0.005 + 0.015 * rng.uniform());
    uint32_t base = (uint32_t)(pos->size() / 3);
    const double sgn[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    for (int corner = 0; corner < 4; ++corner) {
      for (int k = 0; k < 3; ++k) {
        pos->push_back((float)(c[k] + h * (sgn[corner][0] * u[k] + sgn[corner][1] * v[k])));
        nrm->push_back((float)n[k]);
      }
    }
    uint32_t tri[6] = {base, base + 1, base + 2, base, base + 2, base + 3};
    idx->insert(idx->end(), tri, tri + 6);
  }
}

}  // namespace r2
