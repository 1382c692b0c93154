// Stand-in for the NanoVDB bounding box type named by intersect/aabb.hpp
// (test infrastructure).
#ifndef R2_REFSHIM_NANOVDB_H
#define R2_REFSHIM_NANOVDB_H
namespace nanovdb {
struct Vec3R { double v[3]; double operator[](int i) const { return v[i]; } };
struct BBoxR {
  Vec3R lo, hi;
  const Vec3R& min() const { return lo; }
  const Vec3R& max() const { return hi; }
};
}  // namespace nanovdb
#endif
