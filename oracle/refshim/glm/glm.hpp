// Minimal glm-compatible vector/matrix library used ONLY to compile the
// reference's device/host math headers for the host (oracle/ref_kat.cpp,
// test infrastructure).  Written from glm's documented semantics:
// column-major matrices, component-wise vector operators, operator* of
// matrices accumulating column contributions left to right,
// normalize(v) = v * inversesqrt(dot(v, v)) with inversesqrt(x) = 1/sqrt(x).
#ifndef R2_REFSHIM_GLM_HPP
#define R2_REFSHIM_GLM_HPP
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace glm {

typedef int length_t;
enum qualifier { defaultp = 0 };

template <length_t L, typename T, qualifier Q = defaultp> struct vec;

template <typename T, qualifier Q>
struct vec<2, T, Q> {
  T x, y;
  vec() : x(0), y(0) {}
  explicit vec(T s) : x(s), y(s) {}
  vec(T a, T b) : x(a), y(b) {}
  template <typename U> explicit vec(const vec<2, U, Q>& o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)) {}
  template <typename U> vec& operator=(const vec<2, U, Q>& o) { x = static_cast<T>(o.x); y = static_cast<T>(o.y); return *this; }
  T& operator[](length_t i) { return i == 0 ? x : y; }
  const T& operator[](length_t i) const { return i == 0 ? x : y; }
  static constexpr length_t length() { return 2; }
};

template <typename T, qualifier Q>
struct vec<3, T, Q> {
  union { T x; T r; };
  union { T y; T g; };
  union { T z; T b; };
  vec() : x(0), y(0), z(0) {}
  explicit vec(T s) : x(s), y(s), z(s) {}
  vec(T a, T b_, T c) : x(a), y(b_), z(c) {}
  template <typename U> explicit vec(const vec<3, U, Q>& o)
      : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)) {}
  // implicit, as glm's conversions are unless GLM_FORCE_EXPLICIT_CTOR is defined
  template <typename U> vec(const vec<4, U, Q>& o)
      : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)) {}
  template <typename U> vec& operator=(const vec<3, U, Q>& o) {
    x = static_cast<T>(o.x); y = static_cast<T>(o.y); z = static_cast<T>(o.z); return *this;
  }
  vec& operator=(const vec& o) = default;
  vec(const vec& o) = default;
  T& operator[](length_t i) { return i == 0 ? x : (i == 1 ? y : z); }
  const T& operator[](length_t i) const { return i == 0 ? x : (i == 1 ? y : z); }
  static constexpr length_t length() { return 3; }
  vec& operator+=(const vec& o) { x += o.x; y += o.y; z += o.z; return *this; }
  vec& operator-=(const vec& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  vec& operator*=(const vec& o) { x *= o.x; y *= o.y; z *= o.z; return *this; }
  vec& operator*=(T s) { x *= s; y *= s; z *= s; return *this; }
  vec& operator/=(T s) { x /= s; y /= s; z /= s; return *this; }
  vec& operator/=(const vec& o) { x /= o.x; y /= o.y; z /= o.z; return *this; }
};

template <typename T, qualifier Q>
struct vec<4, T, Q> {
  T x, y, z, w;
  vec() : x(0), y(0), z(0), w(0) {}
  explicit vec(T s) : x(s), y(s), z(s), w(s) {}
  vec(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
  vec(const vec<3, T, Q>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
  template <typename U> vec(const vec<3, U, Q>& v, T d)
      : x(static_cast<T>(v.x)), y(static_cast<T>(v.y)), z(static_cast<T>(v.z)), w(d) {}
  template <typename U> explicit vec(const vec<4, U, Q>& o)
      : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)), w(static_cast<T>(o.w)) {}
  T& operator[](length_t i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  const T& operator[](length_t i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  static constexpr length_t length() { return 4; }
};

typedef vec<2, float> vec2;
typedef vec<3, float> vec3;
typedef vec<4, float> vec4;
typedef vec<3, int> ivec3;
typedef vec<3, unsigned int> uvec3;
typedef vec<3, uint8_t> u8vec3;
typedef vec<3, uint16_t> u16vec3;
typedef vec<3, double> dvec3;

// ---- vector operators (component-wise)
#define R2G_BIN(OP)                                                                                      \
  template <typename T, qualifier Q> vec<2, T, Q> operator OP(const vec<2, T, Q>& a, const vec<2, T, Q>& b) { \
    return vec<2, T, Q>(a.x OP b.x, a.y OP b.y);                                                          \
  }                                                                                                      \
  template <typename T, qualifier Q> vec<3, T, Q> operator OP(const vec<3, T, Q>& a, const vec<3, T, Q>& b) { \
    return vec<3, T, Q>(a.x OP b.x, a.y OP b.y, a.z OP b.z);                                              \
  }                                                                                                      \
  template <typename T, qualifier Q> vec<4, T, Q> operator OP(const vec<4, T, Q>& a, const vec<4, T, Q>& b) { \
    return vec<4, T, Q>(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w);                                 \
  }                                                                                                      \
  template <typename T, qualifier Q> vec<2, T, Q> operator OP(const vec<2, T, Q>& a, T s) {              \
    return vec<2, T, Q>(a.x OP s, a.y OP s);                                                              \
  }                                                                                                      \
  template <typename T, qualifier Q> vec<3, T, Q> operator OP(const vec<3, T, Q>& a, T s) {              \
    return vec<3, T, Q>(a.x OP s, a.y OP s, a.z OP s);                                                    \
  }                                                                                                      \
  template <typename T, qualifier Q> vec<4, T, Q> operator OP(const vec<4, T, Q>& a, T s) {              \
    return vec<4, T, Q>(a.x OP s, a.y OP s, a.z OP s, a.w OP s);                                          \
  }                                                                                                      \
  template <typename T, qualifier Q> vec<2, T, Q> operator OP(T s, const vec<2, T, Q>& a) {              \
    return vec<2, T, Q>(s OP a.x, s OP a.y);                                                              \
  }                                                                                                      \
  template <typename T, qualifier Q> vec<3, T, Q> operator OP(T s, const vec<3, T, Q>& a) {              \
    return vec<3, T, Q>(s OP a.x, s OP a.y, s OP a.z);                                                    \
  }                                                                                                      \
  template <typename T, qualifier Q> vec<4, T, Q> operator OP(T s, const vec<4, T, Q>& a) {              \
    return vec<4, T, Q>(s OP a.x, s OP a.y, s OP a.z, s OP a.w);                                          \
  }
R2G_BIN(+)
R2G_BIN(-)
R2G_BIN(*)
R2G_BIN(/)
#undef R2G_BIN

template <typename T, qualifier Q> vec<3, T, Q> operator-(const vec<3, T, Q>& a) { return vec<3, T, Q>(-a.x, -a.y, -a.z); }
template <typename T, qualifier Q> vec<2, T, Q> operator-(const vec<2, T, Q>& a) { return vec<2, T, Q>(-a.x, -a.y); }
template <typename T, qualifier Q> vec<4, T, Q> operator-(const vec<4, T, Q>& a) { return vec<4, T, Q>(-a.x, -a.y, -a.z, -a.w); }
template <typename T, qualifier Q> bool operator==(const vec<3, T, Q>& a, const vec<3, T, Q>& b) {
  return a.x == b.x && a.y == b.y && a.z == b.z;
}
template <typename T, qualifier Q> bool operator!=(const vec<3, T, Q>& a, const vec<3, T, Q>& b) { return !(a == b); }
template <typename T, qualifier Q> bool operator==(const vec<2, T, Q>& a, const vec<2, T, Q>& b) {
  return a.x == b.x && a.y == b.y;
}

// ---- scalar functions
using std::abs;
using std::acos;
using std::atan;
using std::ceil;
using std::cos;
using std::exp;
using std::floor;
using std::log;
using std::round;
using std::sin;
using std::sqrt;
using std::tan;
inline float atan(float y, float x) { return std::atan2(y, x); }
template <typename T> T min(T a, T b) { return (b < a) ? b : a; }
template <typename T> T max(T a, T b) { return (a < b) ? b : a; }
template <typename T> T clamp(T x, T lo, T hi) { return min(max(x, lo), hi); }
template <typename T> bool isinf(T x) { return std::isinf(x); }
template <typename T> bool isnan(T x) { return std::isnan(x); }
inline float radians(float d) { return d * 0.01745329251994329576923690768489f; }
template <typename T> T mix(T a, T b, T t) { return a + t * (b - a); }
inline float inversesqrt(float x) { return 1.0f / std::sqrt(x); }

// ---- vector functions
template <typename T, qualifier Q> T dot(const vec<3, T, Q>& a, const vec<3, T, Q>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename T, qualifier Q> T dot(const vec<2, T, Q>& a, const vec<2, T, Q>& b) { return a.x * b.x + a.y * b.y; }
template <typename T, qualifier Q> T dot(const vec<4, T, Q>& a, const vec<4, T, Q>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}
template <typename T, qualifier Q> vec<3, T, Q> cross(const vec<3, T, Q>& a, const vec<3, T, Q>& b) {
  return vec<3, T, Q>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template <length_t L, typename T, qualifier Q> T length(const vec<L, T, Q>& v) { return std::sqrt(dot(v, v)); }
template <length_t L, typename T, qualifier Q> vec<L, T, Q> normalize(const vec<L, T, Q>& v) {
  return v * (static_cast<T>(1) / std::sqrt(dot(v, v)));
}
template <typename T, qualifier Q> vec<3, T, Q> reflect(const vec<3, T, Q>& i, const vec<3, T, Q>& n) {
  return i - n * dot(n, i) * static_cast<T>(2);
}
#define R2G_MAP3(NAME, EXPR)                                                                         \
  template <typename T, qualifier Q> vec<3, T, Q> NAME(const vec<3, T, Q>& v) {                     \
    return vec<3, T, Q>(EXPR(v.x), EXPR(v.y), EXPR(v.z));                                            \
  }                                                                                                  \
  template <typename T, qualifier Q> vec<4, T, Q> NAME(const vec<4, T, Q>& v) {                     \
    return vec<4, T, Q>(EXPR(v.x), EXPR(v.y), EXPR(v.z), EXPR(v.w));                                 \
  }
R2G_MAP3(abs, std::abs)
R2G_MAP3(floor, std::floor)
R2G_MAP3(ceil, std::ceil)
R2G_MAP3(round, std::round)
R2G_MAP3(sqrt, std::sqrt)
#undef R2G_MAP3
template <typename T, qualifier Q> vec<3, T, Q> min(const vec<3, T, Q>& a, const vec<3, T, Q>& b) {
  return vec<3, T, Q>(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z));
}
template <typename T, qualifier Q> vec<3, T, Q> max(const vec<3, T, Q>& a, const vec<3, T, Q>& b) {
  return vec<3, T, Q>(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z));
}
template <typename T, qualifier Q> vec<3, T, Q> clamp(const vec<3, T, Q>& v, T lo, T hi) {
  return vec<3, T, Q>(clamp(v.x, lo, hi), clamp(v.y, lo, hi), clamp(v.z, lo, hi));
}
template <typename T, qualifier Q> vec<3, bool, Q> isnan(const vec<3, T, Q>& v) {
  return vec<3, bool, Q>(std::isnan(v.x), std::isnan(v.y), std::isnan(v.z));
}
template <typename T, qualifier Q> vec<3, bool, Q> isinf(const vec<3, T, Q>& v) {
  return vec<3, bool, Q>(std::isinf(v.x), std::isinf(v.y), std::isinf(v.z));
}
template <typename T, qualifier Q> vec<3, bool, Q> greaterThanEqual(const vec<3, T, Q>& a, const vec<3, T, Q>& b) {
  return vec<3, bool, Q>(a.x >= b.x, a.y >= b.y, a.z >= b.z);
}
template <qualifier Q> bool any(const vec<3, bool, Q>& v) { return v.x || v.y || v.z; }
template <typename T, qualifier Q> vec<3, T, Q> mix(const vec<3, T, Q>& a, const vec<3, T, Q>& b,
                                                    const vec<3, bool, Q>& s) {
  return vec<3, T, Q>(s.x ? b.x : a.x, s.y ? b.y : a.y, s.z ? b.z : a.z);
}

// ---- matrices (column major): C columns of R-vectors
template <length_t C, length_t R, typename T, qualifier Q = defaultp>
struct mat {
  vec<R, T, Q> c[C];
  mat() {
    for (length_t i = 0; i < C; ++i) c[i] = vec<R, T, Q>(static_cast<T>(0));
  }
  explicit mat(T s) {
    for (length_t i = 0; i < C; ++i) {
      c[i] = vec<R, T, Q>(static_cast<T>(0));
      if (i < R) c[i][i] = s;
    }
  }
  vec<R, T, Q>& operator[](length_t i) { return c[i]; }
  const vec<R, T, Q>& operator[](length_t i) const { return c[i]; }
  // conversion between sizes: copy the overlap, identity elsewhere (implicit,
  // as glm's conversions are unless GLM_FORCE_EXPLICIT_CTOR is defined)
  template <length_t C2, length_t R2> mat(const mat<C2, R2, T, Q>& o) {
    for (length_t i = 0; i < C; ++i) {
      c[i] = vec<R, T, Q>(static_cast<T>(0));
      if (i < R) c[i][i] = static_cast<T>(1);
      for (length_t j = 0; j < R; ++j)
        if (i < C2 && j < R2) c[i][j] = o.c[i][j];
    }
  }
  mat(const vec<R, T, Q>& a, const vec<R, T, Q>& b, const vec<R, T, Q>& d) { c[0] = a; c[1] = b; c[2] = d; }
  mat(const vec<R, T, Q>& a, const vec<R, T, Q>& b, const vec<R, T, Q>& d, const vec<R, T, Q>& e) {
    c[0] = a; c[1] = b; c[2] = d; c[3] = e;
  }
  mat(T a0, T a1, T a2, T b0, T b1, T b2, T c0, T c1, T c2) {
    c[0] = vec<R, T, Q>(a0, a1, a2); c[1] = vec<R, T, Q>(b0, b1, b2); c[2] = vec<R, T, Q>(c0, c1, c2);
  }
  mat& operator+=(const mat& o) { for (length_t i = 0; i < C; ++i) c[i] += o.c[i]; return *this; }
};

typedef mat<3, 3, float> mat3;
typedef mat<4, 4, float> mat4;
typedef mat<4, 3, float> mat4x3;

template <length_t C, length_t R, typename T, qualifier Q>
mat<C, R, T, Q> operator+(const mat<C, R, T, Q>& a, const mat<C, R, T, Q>& b) {
  mat<C, R, T, Q> r;
  for (length_t i = 0; i < C; ++i) r.c[i] = a.c[i] + b.c[i];
  return r;
}
template <length_t C, length_t R, typename T, qualifier Q>
mat<C, R, T, Q> operator*(T s, const mat<C, R, T, Q>& a) {
  mat<C, R, T, Q> r;
  for (length_t i = 0; i < C; ++i) r.c[i] = s * a.c[i];
  return r;
}
template <length_t C, length_t R, typename T, qualifier Q>
mat<C, R, T, Q> operator*(const mat<C, R, T, Q>& a, T s) {
  mat<C, R, T, Q> r;
  for (length_t i = 0; i < C; ++i) r.c[i] = a.c[i] * s;
  return r;
}
// matrix * column vector: sum_k col_k * v[k], left to right.  The vector's
// type is not deduced (glm declares it as the matrix's row_type), so a vec4
// converts to the vec3 a mat3 takes.
template <length_t C, typename T, qualifier Q> struct vec_of { typedef vec<C, T, Q> type; };
template <length_t C, length_t R, typename T, qualifier Q>
vec<R, T, Q> operator*(const mat<C, R, T, Q>& m, const typename vec_of<C, T, Q>::type& v) {
  vec<R, T, Q> r = m.c[0] * v[0];
  for (length_t k = 1; k < C; ++k) r = r + m.c[k] * v[k];
  return r;
}
// matrix * matrix
template <length_t C, length_t K, length_t R, typename T, qualifier Q>
mat<C, R, T, Q> operator*(const mat<K, R, T, Q>& a, const mat<C, K, T, Q>& b) {
  mat<C, R, T, Q> r;
  for (length_t j = 0; j < C; ++j) r.c[j] = a * b.c[j];
  return r;
}

template <typename T, qualifier Q> T determinant(const mat<3, 3, T, Q>& m) {
  return m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) - m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
         m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
}
// inverse through the adjugate (cofactor transpose) divided by the determinant
template <typename T, qualifier Q> mat<3, 3, T, Q> inverse(const mat<3, 3, T, Q>& m) {
  T inv = static_cast<T>(1) / determinant(m);
  mat<3, 3, T, Q> r;
  r[0][0] = +(m[1][1] * m[2][2] - m[2][1] * m[1][2]) * inv;
  r[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * inv;
  r[2][0] = +(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * inv;
  r[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * inv;
  r[1][1] = +(m[0][0] * m[2][2] - m[2][0] * m[0][2]) * inv;
  r[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * inv;
  r[0][2] = +(m[0][1] * m[1][2] - m[1][1] * m[0][2]) * inv;
  r[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * inv;
  r[2][2] = +(m[0][0] * m[1][1] - m[1][0] * m[0][1]) * inv;
  return r;
}
// 4x4 inverse by Gauss-Jordan elimination in double, rounded to T
template <typename T, qualifier Q> mat<4, 4, T, Q> inverse(const mat<4, 4, T, Q>& a) {
  double A[4][8];
  for (int r = 0; r < 4; ++r) {
    for (int c = 0; c < 4; ++c) A[r][c] = a[c][r];
    for (int c = 0; c < 4; ++c) A[r][4 + c] = (r == c) ? 1.0 : 0.0;
  }
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
    if (piv != c)
      for (int k = 0; k < 8; ++k) { double t = A[c][k]; A[c][k] = A[piv][k]; A[piv][k] = t; }
    double p = A[c][c];
    for (int k = 0; k < 8; ++k) A[c][k] /= p;
    for (int r = 0; r < 4; ++r) {
      if (r == c) continue;
      double f = A[r][c];
      for (int k = 0; k < 8; ++k) A[r][k] -= f * A[c][k];
    }
  }
  mat<4, 4, T, Q> r;
  for (int row = 0; row < 4; ++row)
    for (int c = 0; c < 4; ++c) r[c][row] = static_cast<T>(A[row][4 + c]);
  return r;
}

namespace detail {
// IEEE binary16 conversion (round to nearest even), from the format definition.
inline uint16_t toFloat16(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
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
inline float toFloat32(uint16_t h) {
  uint32_t sign = ((uint32_t)h & 0x8000u) << 16, e = (h >> 10) & 0x1Fu, m = h & 0x3FFu, x;
  if (e == 0) {
    float f = (float)m * (1.0f / 16777216.0f);
    std::memcpy(&x, &f, 4);
    x |= sign;
  } else if (e == 31) {
    x = sign | 0x7F800000u | (m << 13);
  } else {
    x = sign | ((e + 112u) << 23) | (m << 13);
  }
  float f;
  std::memcpy(&f, &x, 4);
  return f;
}
}  // namespace detail

}  // namespace glm

#endif
