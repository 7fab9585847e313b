// oracle/om.h -- TEST INFRASTRUCTURE (the oracle). CPU restatement of the vector math the
// reference step runs on. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
// may use anything under oracle/; the product never links it.
//
// The reference does its math through glam 0.27 (Vec3 / Mat3A / Quat, `libm` feature;
// Cargo.lock:998-1000, Cargo.toml:37), a crate that is not vendored under the reference tree.
// What is restated here is glam's formulas, in plain f32 with no FMA contraction (build flag
// -ffp-contract=off): Vec3 / Mat3 scalar, Quat in the lane order of its SSE2 paths (below). The
// operation order is the one the oracle and the CUDA kernels share, so the two agree bit for bit,
// and with these forms the oracle reproduces the reference's own golden bits for its
// distance-joint scenes (distance_bits_test.rs:50-57).
//
// Transcendentals (sin, cos, exp) are the project's own: Cody-Waite argument reduction with
// split constants derived from pi/2 and ln 2 to 80 digits, then Taylor polynomials evaluated
// in double, rounded once to f32. The same code runs on the GPU, so results match bit for bit.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace om {

struct V3 { float x, y, z; };
struct Q4 { float x, y, z, w; };
// Column-major 3x3 (glam Mat3A): c0, c1, c2 are the columns.
struct M3 { V3 c0, c1, c2; };

static inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
static inline V3 splat(float s) { return V3{s, s, s}; }
static inline V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 mul(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
static inline V3 mulv(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
static inline V3 divs(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
static inline V3 neg(V3 a) { return V3{-a.x, -a.y, -a.z}; }
static inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
  return V3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
static inline float len2(V3 a) { return dot(a, a); }
static inline float len(V3 a) { return std::sqrt(dot(a, a)); }
static inline V3 vabs(V3 a) { return V3{std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
// Rust f32::min / f32::max (and glam's scalar Vec3::min/max, which call them): IEEE
// minNum/maxNum, a NaN operand is ignored.
static inline float rmin(float a, float b) { return std::fmin(a, b); }
static inline float rmax(float a, float b) { return std::fmax(a, b); }
static inline V3 vmin(V3 a, V3 b) { return V3{rmin(a.x, b.x), rmin(a.y, b.y), rmin(a.z, b.z)}; }
static inline V3 vmax(V3 a, V3 b) { return V3{rmax(a.x, b.x), rmax(a.y, b.y), rmax(a.z, b.z)}; }
static inline bool fin(float x) { return std::isfinite(x); }
static inline bool vfin(V3 a) { return fin(a.x) && fin(a.y) && fin(a.z); }
static inline bool qfin(Q4 q) { return fin(q.x) && fin(q.y) && fin(q.z) && fin(q.w); }
static inline float fin0(float x) { return fin(x) ? x : 0.0f; }
static inline V3 fin_v(V3 a) { return V3{fin0(a.x), fin0(a.y), fin0(a.z)}; }
static inline bool veq(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
static inline bool vzero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
// Rust f32::clamp
static inline float clampf(float x, float lo, float hi) { if (x < lo) x = lo; if (x > hi) x = hi; return x; }
// Vec3::normalize: self * (1 / length)
static inline V3 normalize(V3 a) { float r = 1.0f / len(a); return mul(a, r); }
// Vec3::normalize_or_zero
static inline V3 normalize_or_zero(V3 a) {
  float r = 1.0f / len(a);
  if (fin(r) && r > 0.0f) return mul(a, r);
  return V3{0, 0, 0};
}
// Vec3::clamp_length_max
static inline V3 clamp_length_max(V3 a, float m) {
  float l2 = len2(a);
  if (l2 > m * m) { float l = std::sqrt(l2); V3 d = divs(a, l); return mul(d, m); }
  return a;
}

// ---- quaternions (x, y, z, w) ----
// glam's Quat is an SSE2 type on x86_64, where the reference runs, so its product and norm follow
// the lane order of glam's SSE2 paths (Quat::mul_quat after rtm's quat_mul, dot4, Vec4::normalize):
// the Hamilton product lane-wise as (w0 b + x0 b1) + (y0 b2 + z0 b3), b1..b3 the signed lane
// permutations of b; the 4-lane dot as (xx + zz) + (yy + ww); normalize as a division by the
// length. These forms reproduce the reference's golden bits of distance_bits_test.rs:50-57
// (tests/test_oracle_golden.py); the scalar forms do not.
static inline Q4 qmul(Q4 a, Q4 b) {
  return Q4{(a.w * b.x + a.x * b.w) + (a.y * b.z - a.z * b.y),
            (a.w * b.y - a.x * b.z) + (a.y * b.w + a.z * b.x),
            (a.w * b.z + a.x * b.y) + (-(a.y * b.x) + a.z * b.w),
            (a.w * b.w - a.x * b.x) + (-(a.y * b.y) - a.z * b.z)};
}
static inline Q4 qconj(Q4 q) { return Q4{-q.x, -q.y, -q.z, q.w}; }
static inline Q4 qneg(Q4 q) { return Q4{-q.x, -q.y, -q.z, -q.w}; }
static inline float qdot(Q4 a, Q4 b) { return (a.x * b.x + a.z * b.z) + (a.y * b.y + a.w * b.w); }
static inline Q4 qscale(Q4 q, float s) { return Q4{q.x * s, q.y * s, q.z * s, q.w * s}; }
static inline Q4 qnormalize(Q4 q) {
  float l = std::sqrt(qdot(q, q));
  return Q4{q.x / l, q.y / l, q.z / l, q.w / l};
}
static inline bool qeq(Q4 a, Q4 b) { return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w; }
// Quat * Vec3: v (w^2 - b.b) + b (2 v.b) + (b x v)(2 w)
static inline V3 qrot(Q4 q, V3 v) {
  V3 b = V3{q.x, q.y, q.z};
  float b2 = dot(b, b);
  V3 t1 = mul(v, q.w * q.w - b2);
  V3 t2 = mul(b, dot(v, b) * 2.0f);
  V3 t3 = mul(cross(b, v), q.w * 2.0f);
  return add(add(t1, t2), t3);
}

// ---- 3x3 matrices ----
static inline M3 mzero() { return M3{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}; }
static inline M3 mdiag(V3 d) { return M3{{d.x, 0, 0}, {0, d.y, 0}, {0, 0, d.z}}; }
// Mat3A * Vec3: c0 v.x + c1 v.y + c2 v.z
static inline V3 mvec(const M3& m, V3 v) {
  return add(add(mul(m.c0, v.x), mul(m.c1, v.y)), mul(m.c2, v.z));
}
static inline M3 mmul(const M3& a, const M3& b) { return M3{mvec(a, b.c0), mvec(a, b.c1), mvec(a, b.c2)}; }
static inline M3 mtranspose(const M3& m) {
  return M3{{m.c0.x, m.c1.x, m.c2.x}, {m.c0.y, m.c1.y, m.c2.y}, {m.c0.z, m.c1.z, m.c2.z}};
}
static inline M3 msub(const M3& a, const M3& b) { return M3{sub(a.c0, b.c0), sub(a.c1, b.c1), sub(a.c2, b.c2)}; }
static inline bool mis_zero(const M3& m) { return vzero(m.c0) && vzero(m.c1) && vzero(m.c2); }
static inline float mdet(const M3& m) { return dot(m.c2, cross(m.c0, m.c1)); }
static inline M3 minverse(const M3& m) {
  V3 t0 = cross(m.c1, m.c2), t1 = cross(m.c2, m.c0), t2 = cross(m.c0, m.c1);
  float det = dot(m.c2, t2);
  float inv = 1.0f / det;
  return mtranspose(M3{mul(t0, inv), mul(t1, inv), mul(t2, inv)});
}
// Mat3::from_quat
static inline M3 mfrom_quat(Q4 q) {
  float x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
  float xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
  float yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
  float wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
  return M3{{1.0f - (yy + zz), xy + wz, xz - wy},
            {xy - wz, 1.0f - (xx + zz), yz + wx},
            {xz + wy, yz - wx, 1.0f - (xx + yy)}};
}

// ---- portable transcendentals (project's own; identical on the GPU) ----
static const double kTwoOverPi = 0x1.45f306dc9c883p-1;
static const double kPio2_1 = 0x1.921fb54400000p+0;
static const double kPio2_2 = 0x1.0b4611a600000p-34;
static const double kPio2_3 = 0x1.3198a2e037073p-69;

// Taylor series of sin and cos about 0, |r| <= pi/4 (+ reduction slack): terms through r^19 / r^18.
static inline double sin_poly(double r) {
  double r2 = r * r;
  double p = -1.0 / 121645100408832000.0;           // -1/19!
  p = p * r2 + 1.0 / 355687428096000.0;              // 1/17!
  p = p * r2 - 1.0 / 1307674368000.0;                // -1/15!
  p = p * r2 + 1.0 / 6227020800.0;                   // 1/13!
  p = p * r2 - 1.0 / 39916800.0;                     // -1/11!
  p = p * r2 + 1.0 / 362880.0;                       // 1/9!
  p = p * r2 - 1.0 / 5040.0;                         // -1/7!
  p = p * r2 + 1.0 / 120.0;                          // 1/5!
  p = p * r2 - 1.0 / 6.0;                            // -1/3!
  return r + (r * r2) * p;
}
static inline double cos_poly(double r) {
  double r2 = r * r;
  double p = 1.0 / 6402373705728000.0;               // 1/18!
  p = p * r2 - 1.0 / 20922789888000.0;               // -1/16!
  p = p * r2 + 1.0 / 87178291200.0;                  // 1/14!
  p = p * r2 - 1.0 / 479001600.0;                    // -1/12!
  p = p * r2 + 1.0 / 3628800.0;                      // 1/10!
  p = p * r2 - 1.0 / 40320.0;                        // -1/8!
  p = p * r2 + 1.0 / 720.0;                          // 1/6!
  p = p * r2 - 1.0 / 24.0;                           // -1/4!
  p = p * r2 + 0.5;                                  // 1/2!
  return 1.0 - r2 * p;
}
// sin and cos of an f32 angle, each rounded once to f32.
static inline void sincosf_rp(float xf, float* s, float* c) {
  double x = (double)xf;
  if (!std::isfinite(x)) { *s = NAN; *c = NAN; return; }
  double k = std::floor(x * kTwoOverPi + 0.5);
  double r = ((x - k * kPio2_1) - k * kPio2_2) - k * kPio2_3;
  long long q = (long long)k;
  int qi = (int)(q & 3);
  double sr = sin_poly(r), cr = cos_poly(r);
  double sv, cv;
  switch (qi) {
    case 0: sv = sr; cv = cr; break;
    case 1: sv = cr; cv = -sr; break;
    case 2: sv = -sr; cv = -cr; break;
    default: sv = -cr; cv = sr; break;
  }
  *s = (float)sv; *c = (float)cv;
}
// exp of an f32, rounded once to f32: x = (32 m + j) ln2/32 + r with |r| <= ln2/64, e^x = 2^m 2^(j/32) e^r;
// 2^(j/32) the double nearest it (computed with 80-digit decimal arithmetic), e^r - 1 by its
// Taylor series through r^5 (error below 3e-15).
static const double kExp2_32[32] = {
  0x1.0000000000000p+0, 0x1.059b0d3158574p+0, 0x1.0b5586cf9890fp+0, 0x1.11301d0125b51p+0,
  0x1.172b83c7d517bp+0, 0x1.1d4873168b9aap+0, 0x1.2387a6e756238p+0, 0x1.29e9df51fdee1p+0,
  0x1.306fe0a31b715p+0, 0x1.371a7373aa9cbp+0, 0x1.3dea64c123422p+0, 0x1.44e086061892dp+0,
  0x1.4bfdad5362a27p+0, 0x1.5342b569d4f82p+0, 0x1.5ab07dd485429p+0, 0x1.6247eb03a5585p+0,
  0x1.6a09e667f3bcdp+0, 0x1.71f75e8ec5f74p+0, 0x1.7a11473eb0187p+0, 0x1.82589994cce13p+0,
  0x1.8ace5422aa0dbp+0, 0x1.93737b0cdc5e5p+0, 0x1.9c49182a3f090p+0, 0x1.a5503b23e255dp+0,
  0x1.ae89f995ad3adp+0, 0x1.b7f76f2fb5e47p+0, 0x1.c199bdd85529cp+0, 0x1.cb720dcef9069p+0,
  0x1.d5818dcfba487p+0, 0x1.dfc97337b9b5fp+0, 0x1.ea4afa2a490dap+0, 0x1.f50765b6e4540p+0
};
static inline float expf_rp(float xf) {
  double x = (double)xf;
  if (std::isnan(x)) return NAN;
  if (x > 89.0) return INFINITY;
  if (x < -104.0) return 0.0f;
  double k = std::floor(x * 0x1.71547652b82fep+5 + 0.5);               // 32 / ln2
  double r = (x - k * 0x1.62e42fef00000p-6) - k * 0x1.473de6af278edp-39;  // ln2/32, split
  long long ki = (long long)k;
  int j = (int)(ki & 31), m = (int)((ki - j) / 32);
  double r2 = r * r;
  double q = r + (r2 * (0.5 + r * (1.0 / 6.0)) + (r2 * r2) * (1.0 / 24.0 + r * (1.0 / 120.0)));
  double t = kExp2_32[j];
  double p = t + t * q;
  return (float)std::ldexp(p, m);
}

// Quat::from_axis_angle(axis, angle): (axis sin(angle/2), cos(angle/2))
static inline Q4 qfrom_axis_angle(V3 axis, float angle) {
  float s, c;
  sincosf_rp(angle * 0.5f, &s, &c);
  V3 v = mul(axis, s);
  return Q4{v.x, v.y, v.z, c};
}

// atan of a non-negative double: 1/x for x > 1, then two half-angle reductions
// t -> t / (1 + sqrt(1 + t^2)) (atan t = 2 atan of the result) leave |t| <= tan(pi/16) ~ 0.199,
// then the Taylor series t - t^3/3 + ... through t^27 and the sum times 4.
static const double kPio2Hi = 0x1.921fb54442d18p+0;
static const double kPio2Lo = 0x1.1a62633145c07p-54;
static inline double atan_d(double x) {
  bool inv = x > 1.0;
  if (inv) x = 1.0 / x;
  double t = x / (1.0 + std::sqrt(1.0 + x * x));
  t = t / (1.0 + std::sqrt(1.0 + t * t));
  double z = t * t;
  double p = -1.0 / 27.0;
  p = p * z + 1.0 / 25.0;
  p = p * z - 1.0 / 23.0;
  p = p * z + 1.0 / 21.0;
  p = p * z - 1.0 / 19.0;
  p = p * z + 1.0 / 17.0;
  p = p * z - 1.0 / 15.0;
  p = p * z + 1.0 / 13.0;
  p = p * z - 1.0 / 11.0;
  p = p * z + 1.0 / 9.0;
  p = p * z - 1.0 / 7.0;
  p = p * z + 1.0 / 5.0;
  p = p * z - 1.0 / 3.0;
  double a = 4.0 * (t + (t * z) * p);
  if (inv) a = (kPio2Hi - a) + kPio2Lo;
  return a;
}
// f32 atan2 with IEEE's special cases, evaluated in double and rounded once.
static inline float atan2f_rp(float yf, float xf) {
  if (std::isnan(yf) || std::isnan(xf)) return NAN;
  const double pi = 2.0 * kPio2Hi;
  double y = (double)yf, x = (double)xf, a;
  if (yf == 0.0f) a = std::signbit(xf) ? pi : 0.0;
  else if (std::isinf(xf) && std::isinf(yf)) a = xf > 0.0f ? 0.5 * kPio2Hi : 1.5 * kPio2Hi;
  else if (std::isinf(xf)) a = xf > 0.0f ? 0.0 : pi;
  else if (xf == 0.0f || std::isinf(yf)) a = kPio2Hi;
  else {
    a = atan_d(std::fabs(y) / std::fabs(x));
    if (xf < 0.0f) a = pi - a;
  }
  return (float)(std::signbit(yf) ? -a : a);
}
// f32 acos of d in [0, 1]: 2 atan(sqrt((1 - d) / (1 + d))), rounded once.
static inline float acosf_unit_rp(float df) {
  double d = (double)df;
  return (float)(2.0 * atan_d(std::sqrt((1.0 - d) / (1.0 + d))));
}

// ---- determinism helpers (riftphys-core/src/det.rs, determinism.rs) ----
// q6 (det.rs:11-17): non-finite -> 0; round(x / 1e-6) * 1e-6
static inline float q6(float x) {
  if (!fin(x)) return 0.0f;
  return std::round(x / 1.0e-6f) * 1.0e-6f;
}
// qf32 (determinism.rs:57-65) at the default 1e-6 step: non-finite -> NaN
static inline float qf32(float x) {
  if (!fin(x)) return NAN;
  return std::round(x / 1.0e-6f) * 1.0e-6f;
}
// materials::quantize (materials.rs:319): round(x * 1e6) * 1e-6
static inline float quantize_mat(float x) { return std::round(x * 1.0e6f) * 1.0e-6f; }
// sort_key6 (det.rs:25-29)
static inline int64_t sort_key6(float x) {
  if (std::isnan(x)) return INT64_MAX;
  double k = std::round((double)x * 1.0e6);
  if (k >= 9223372036854775807.0) return INT64_MAX;
  if (k <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)k;
}
// canon_f32_bits (hash.rs:24-34)
static inline uint32_t canon_bits(float x) {
  if (!fin(x)) return 0x7fc00000u;
  uint32_t b; std::memcpy(&b, &x, 4);
  return b == 0x80000000u ? 0u : b;
}
static inline float signum(float x) {
  if (std::isnan(x)) return NAN;
  return std::signbit(x) ? -1.0f : 1.0f;
}

}  // namespace om
