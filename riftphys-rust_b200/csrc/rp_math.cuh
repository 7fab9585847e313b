// rp_math.cuh -- f32 vector math for the step kernels (and the host code that must agree with
// them bit for bit: mass properties, pose sanitation).
//
// The reference computes with glam 0.27's Vec3 / Mat3A / Quat (Cargo.lock:998-1000). Each
// function below evaluates glam's published scalar formula in a fixed order of IEEE f32
// operations; the library is built with --fmad=false (device) and -ffp-contract=off (host), so
// no multiply-add is fused and every result is reproducible across the CPU and the GPU.
// sin, cos and exp are the project's own (Cody-Waite reduction with split constants derived
// from pi/2 and ln 2 to 80 digits; Taylor polynomials in double; one rounding to f32), because
// CUDA's and libm's versions differ in the last ulp.
#pragma once
#include <cstdint>
#include <cstring>
#include <math.h>

#ifdef __CUDACC__
#define RP_HD __host__ __device__ __forceinline__
#else
#define RP_HD inline
#endif

namespace rp {

// Collider shapes (riftphys-geom/src/shape.rs:7-14); triangles come only from the heightfield.
enum : uint32_t { SH_SPHERE = 0, SH_BOX = 1, SH_CAPSULE = 2, SH_TRIANGLE = 3 };

struct f3 { float x, y, z; };
struct q4 { float x, y, z, w; };
struct m3 { f3 c0, c1, c2; };  // column-major (glam Mat3A)

RP_HD f3 mk3(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
RP_HD q4 mkq(float x, float y, float z, float w) { q4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r; }
RP_HD f3 splat(float s) { return mk3(s, s, s); }
RP_HD f3 operator+(f3 a, f3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
RP_HD f3 operator-(f3 a, f3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
RP_HD f3 operator*(f3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
RP_HD f3 operator/(f3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
RP_HD f3 operator-(f3 a) { return mk3(-a.x, -a.y, -a.z); }
RP_HD float dot(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
RP_HD f3 cross(f3 a, f3 b) { return mk3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }
RP_HD float len2(f3 a) { return dot(a, a); }
RP_HD float len(f3 a) { return sqrtf(dot(a, a)); }
RP_HD f3 vabs(f3 a) { return mk3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
// Rust f32::min / f32::max (IEEE minNum / maxNum: a NaN operand is ignored), as fminf / fmaxf
RP_HD float rmin(float a, float b) { return fminf(a, b); }
RP_HD float rmax(float a, float b) { return fmaxf(a, b); }
RP_HD f3 vmin(f3 a, f3 b) { return mk3(rmin(a.x, b.x), rmin(a.y, b.y), rmin(a.z, b.z)); }
RP_HD f3 vmax(f3 a, f3 b) { return mk3(rmax(a.x, b.x), rmax(a.y, b.y), rmax(a.z, b.z)); }
RP_HD bool fin(float x) { return isfinite(x); }
RP_HD bool vfin(f3 a) { return fin(a.x) && fin(a.y) && fin(a.z); }
RP_HD bool qfin(q4 q) { return fin(q.x) && fin(q.y) && fin(q.z) && fin(q.w); }
RP_HD float fin0(float x) { return fin(x) ? x : 0.0f; }
RP_HD f3 fin_v(f3 a) { return mk3(fin0(a.x), fin0(a.y), fin0(a.z)); }
RP_HD bool veq(f3 a, f3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
RP_HD bool vzero(f3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
RP_HD float clampf(float x, float lo, float hi) { if (x < lo) x = lo; if (x > hi) x = hi; return x; }
RP_HD f3 normalize(f3 a) { float r = 1.0f / len(a); return a * r; }
RP_HD f3 normalize_or_zero(f3 a) {
  float r = 1.0f / len(a);
  if (fin(r) && r > 0.0f) return a * r;
  return mk3(0, 0, 0);
}
RP_HD f3 clamp_length_max(f3 a, float m) {
  float l2 = len2(a);
  if (l2 > m * m) { float l = sqrtf(l2); f3 d = a / l; return d * m; }
  return a;
}

// glam's Quat is an SSE2 type on x86_64, where the reference runs; its product and norm are
// restated in the lane order of those SSE2 paths (pinned by the reference's golden bits of
// distance_bits_test.rs): the Hamilton product lane-wise as (w0 b + x0 b1) + (y0 b2 + z0 b3), b1..b3
// the signed lane permutations of b; the 4-lane dot as (xx + zz) + (yy + ww); normalize as a
// division by the length.
RP_HD q4 qmul(q4 a, q4 b) {
  return mkq((a.w * b.x + a.x * b.w) + (a.y * b.z - a.z * b.y),
             (a.w * b.y - a.x * b.z) + (a.y * b.w + a.z * b.x),
             (a.w * b.z + a.x * b.y) + (-(a.y * b.x) + a.z * b.w),
             (a.w * b.w - a.x * b.x) + (-(a.y * b.y) - a.z * b.z));
}
RP_HD q4 qconj(q4 q) { return mkq(-q.x, -q.y, -q.z, q.w); }
RP_HD q4 qneg(q4 q) { return mkq(-q.x, -q.y, -q.z, -q.w); }
RP_HD float qdot(q4 a, q4 b) { return (a.x * b.x + a.z * b.z) + (a.y * b.y + a.w * b.w); }
RP_HD q4 qscale(q4 q, float s) { return mkq(q.x * s, q.y * s, q.z * s, q.w * s); }
RP_HD q4 qnormalize(q4 q) {
  float l = sqrtf(qdot(q, q));
  return mkq(q.x / l, q.y / l, q.z / l, q.w / l);
}
RP_HD bool qeq(q4 a, q4 b) { return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w; }
RP_HD f3 qrot(q4 q, f3 v) {
  f3 b = mk3(q.x, q.y, q.z);
  float b2 = dot(b, b);
  f3 t1 = v * (q.w * q.w - b2);
  f3 t2 = b * (dot(v, b) * 2.0f);
  f3 t3 = cross(b, v) * (q.w * 2.0f);
  return (t1 + t2) + t3;
}
RP_HD q4 qident() { return mkq(0, 0, 0, 1); }
// Bodies::fin_q (riftphys-dynamics/src/dynamics.rs:15-20): finite, normalised, w >= 0
RP_HD q4 fin_q(q4 q) {
  if (!qfin(q)) return qident();
  q4 qq = qnormalize(q);
  if (!qfin(qq)) return qident();
  if (qq.w < 0.0f) qq = qneg(qq);
  return qq;
}

RP_HD m3 mzero() { m3 m; m.c0 = mk3(0, 0, 0); m.c1 = mk3(0, 0, 0); m.c2 = mk3(0, 0, 0); return m; }
RP_HD m3 mdiag(f3 d) { m3 m; m.c0 = mk3(d.x, 0, 0); m.c1 = mk3(0, d.y, 0); m.c2 = mk3(0, 0, d.z); return m; }
RP_HD m3 mcols(f3 a, f3 b, f3 c) { m3 m; m.c0 = a; m.c1 = b; m.c2 = c; return m; }
RP_HD f3 mvec(const m3& m, f3 v) { return ((m.c0 * v.x) + (m.c1 * v.y)) + (m.c2 * v.z); }
RP_HD m3 mmul(const m3& a, const m3& b) { return mcols(mvec(a, b.c0), mvec(a, b.c1), mvec(a, b.c2)); }
RP_HD m3 mtranspose(const m3& m) {
  return mcols(mk3(m.c0.x, m.c1.x, m.c2.x), mk3(m.c0.y, m.c1.y, m.c2.y), mk3(m.c0.z, m.c1.z, m.c2.z));
}
RP_HD m3 msub(const m3& a, const m3& b) { return mcols(a.c0 - b.c0, a.c1 - b.c1, a.c2 - b.c2); }
RP_HD float mdet(const m3& m) { return dot(m.c2, cross(m.c0, m.c1)); }
RP_HD m3 minverse(const m3& m) {
  f3 t0 = cross(m.c1, m.c2), t1 = cross(m.c2, m.c0), t2 = cross(m.c0, m.c1);
  float det = dot(m.c2, t2);
  float inv = 1.0f / det;
  return mtranspose(mcols(t0 * inv, t1 * inv, t2 * inv));
}
RP_HD m3 mfrom_quat(q4 q) {
  float x2 = q.x + q.x, y2 = q.y + q.y, z2 = q.z + q.z;
  float xx = q.x * x2, xy = q.x * y2, xz = q.x * z2;
  float yy = q.y * y2, yz = q.y * z2, zz = q.z * z2;
  float wx = q.w * x2, wy = q.w * y2, wz = q.w * z2;
  return mcols(mk3(1.0f - (yy + zz), xy + wz, xz - wy),
               mk3(xy - wz, 1.0f - (xx + zz), yz + wx),
               mk3(xz + wy, yz - wx, 1.0f - (xx + yy)));
}
// R * I_local * R^T
RP_HD m3 world_inertia(q4 q, const m3& il) { m3 r = mfrom_quat(q); return mmul(mmul(r, il), mtranspose(r)); }

// ---- the project's sin / cos / exp (see header comment)
#define RP_TWO_OVER_PI 0x1.45f306dc9c883p-1
#define RP_PIO2_1 0x1.921fb54400000p+0
#define RP_PIO2_2 0x1.0b4611a600000p-34
#define RP_PIO2_3 0x1.3198a2e037073p-69

RP_HD double rp_sin_poly(double r) {
  double r2 = r * r;
  double p = -1.0 / 121645100408832000.0;
  p = p * r2 + 1.0 / 355687428096000.0;
  p = p * r2 - 1.0 / 1307674368000.0;
  p = p * r2 + 1.0 / 6227020800.0;
  p = p * r2 - 1.0 / 39916800.0;
  p = p * r2 + 1.0 / 362880.0;
  p = p * r2 - 1.0 / 5040.0;
  p = p * r2 + 1.0 / 120.0;
  p = p * r2 - 1.0 / 6.0;
  return r + (r * r2) * p;
}
RP_HD double rp_cos_poly(double r) {
  double r2 = r * r;
  double p = 1.0 / 6402373705728000.0;
  p = p * r2 - 1.0 / 20922789888000.0;
  p = p * r2 + 1.0 / 87178291200.0;
  p = p * r2 - 1.0 / 479001600.0;
  p = p * r2 + 1.0 / 3628800.0;
  p = p * r2 - 1.0 / 40320.0;
  p = p * r2 + 1.0 / 720.0;
  p = p * r2 - 1.0 / 24.0;
  p = p * r2 + 0.5;
  return 1.0 - r2 * p;
}
RP_HD void sincos_rp(float xf, float* s, float* c) {
  double x = (double)xf;
  if (!isfinite(x)) { *s = NAN; *c = NAN; return; }
  double k = floor(x * RP_TWO_OVER_PI + 0.5);
  double r = ((x - k * RP_PIO2_1) - k * RP_PIO2_2) - k * RP_PIO2_3;
  long long q = (long long)k;
  int qi = (int)(q & 3);
  double sr = rp_sin_poly(r), cr = rp_cos_poly(r);
  double sv, cv;
  if (qi == 0) { sv = sr; cv = cr; }
  else if (qi == 1) { sv = cr; cv = -sr; }
  else if (qi == 2) { sv = -sr; cv = -cr; }
  else { sv = -cr; cv = sr; }
  *s = (float)sv; *c = (float)cv;
}
// Unit of the learned warm start's impulses: a row's effective mass times 9.81 m/s^2 / 60 Hz (the
// impulse that holds the row's mass against gravity for one tick), written as one f32 constant.
constexpr float kImpulseUnit = 0.1635f;
// exp: x = (32 m + j) ln2/32 + r with |r| <= ln2/64, so e^x = 2^m 2^(j/32) e^r; 2^(j/32) from the
// table below (each entry the double nearest 2^(j/32), computed with 80-digit decimal arithmetic),
// e^r - 1 from its Taylor series through r^5 (error below 3e-15), evaluated in double and rounded
// once to f32. Over every seventh f32 in [-104, 0] it returns the bits of the degree-14 series on
// |r| <= ln2/2 that it replaced, with a shorter dependent chain (the friction law calls it once per
// row update).
#define RP_EXP2_32_TABLE { \
  0x1.0000000000000p+0, 0x1.059b0d3158574p+0, 0x1.0b5586cf9890fp+0, 0x1.11301d0125b51p+0, \
  0x1.172b83c7d517bp+0, 0x1.1d4873168b9aap+0, 0x1.2387a6e756238p+0, 0x1.29e9df51fdee1p+0, \
  0x1.306fe0a31b715p+0, 0x1.371a7373aa9cbp+0, 0x1.3dea64c123422p+0, 0x1.44e086061892dp+0, \
  0x1.4bfdad5362a27p+0, 0x1.5342b569d4f82p+0, 0x1.5ab07dd485429p+0, 0x1.6247eb03a5585p+0, \
  0x1.6a09e667f3bcdp+0, 0x1.71f75e8ec5f74p+0, 0x1.7a11473eb0187p+0, 0x1.82589994cce13p+0, \
  0x1.8ace5422aa0dbp+0, 0x1.93737b0cdc5e5p+0, 0x1.9c49182a3f090p+0, 0x1.a5503b23e255dp+0, \
  0x1.ae89f995ad3adp+0, 0x1.b7f76f2fb5e47p+0, 0x1.c199bdd85529cp+0, 0x1.cb720dcef9069p+0, \
  0x1.d5818dcfba487p+0, 0x1.dfc97337b9b5fp+0, 0x1.ea4afa2a490dap+0, 0x1.f50765b6e4540p+0 }
#ifdef __CUDA_ARCH__
static __device__ const double rp_exp2_32[32] = RP_EXP2_32_TABLE;
#else
static const double rp_exp2_32[32] = RP_EXP2_32_TABLE;
#endif
#define RP_32_OVER_LN2 0x1.71547652b82fep+5
#define RP_LN2_32_HI 0x1.62e42fef00000p-6  // ln2/32 split: k * HI is exact for |k| < 2^20
#define RP_LN2_32_LO 0x1.473de6af278edp-39
RP_HD float exp_rp(float xf) {
  double x = (double)xf;
  if (isnan(x)) return NAN;
  if (x > 89.0) return INFINITY;
  if (x < -104.0) return 0.0f;
  double k = floor(x * RP_32_OVER_LN2 + 0.5);
  double r = (x - k * RP_LN2_32_HI) - k * RP_LN2_32_LO;
  long long ki = (long long)k;
  int j = (int)(ki & 31), m = (int)((ki - j) / 32);
  double r2 = r * r;
  double q = r + (r2 * (0.5 + r * (1.0 / 6.0)) + (r2 * r2) * (1.0 / 24.0 + r * (1.0 / 120.0)));
  double t = rp_exp2_32[j];
  double p = t + t * q;
  // p * 2^m is exact (m in [-150, 128] keeps 2^m a normal double): the value ldexp gives
  long long eb = (long long)(m + 1023) << 52;
  double two_m;
  memcpy(&two_m, &eb, 8);
  return (float)(p * two_m);
}
// atan of a non-negative double: 1/x for x > 1, two half-angle reductions
// t -> t / (1 + sqrt(1 + t^2)) to |t| <= tan(pi/16), the Taylor series through t^27, times 4.
#define RP_PIO2_HI 0x1.921fb54442d18p+0
#define RP_PIO2_LO 0x1.1a62633145c07p-54
RP_HD double atan_d(double x) {
  bool inv = x > 1.0;
  if (inv) x = 1.0 / x;
  double t = x / (1.0 + sqrt(1.0 + x * x));
  t = t / (1.0 + sqrt(1.0 + t * t));
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
  if (inv) a = (RP_PIO2_HI - a) + RP_PIO2_LO;
  return a;
}
// f32 atan2 with IEEE's special cases, evaluated in double and rounded once.
RP_HD float atan2_rp(float yf, float xf) {
  if (isnan(yf) || isnan(xf)) return NAN;
  const double pi = 2.0 * RP_PIO2_HI;
  double y = (double)yf, x = (double)xf, a;
  if (yf == 0.0f) a = signbit(xf) ? pi : 0.0;
  else if (isinf(xf) && isinf(yf)) a = xf > 0.0f ? 0.5 * RP_PIO2_HI : 1.5 * RP_PIO2_HI;
  else if (isinf(xf)) a = xf > 0.0f ? 0.0 : pi;
  else if (xf == 0.0f || isinf(yf)) a = RP_PIO2_HI;
  else {
    a = atan_d(fabs(y) / fabs(x));
    if (xf < 0.0f) a = pi - a;
  }
  return (float)(signbit(yf) ? -a : a);
}
// f32 acos of d in [0, 1]: 2 atan(sqrt((1 - d) / (1 + d))), rounded once.
RP_HD float acos_unit_rp(float df) {
  double d = (double)df;
  return (float)(2.0 * atan_d(sqrt((1.0 - d) / (1.0 + d))));
}
RP_HD q4 qfrom_axis_angle(f3 axis, float angle) {
  float s, c;
  sincos_rp(angle * 0.5f, &s, &c);
  f3 v = axis * s;
  return mkq(v.x, v.y, v.z, c);
}

// ---- determinism helpers (riftphys-core/src/det.rs, determinism.rs, hash.rs)
RP_HD float q6(float x) { if (!fin(x)) return 0.0f; return roundf(x / 1.0e-6f) * 1.0e-6f; }
RP_HD float qf32(float x) { if (!fin(x)) return NAN; return roundf(x / 1.0e-6f) * 1.0e-6f; }
RP_HD float quantize_mat(float x) { return roundf(x * 1.0e6f) * 1.0e-6f; }
RP_HD long long sort_key6(float x) {
  if (isnan(x)) return 9223372036854775807LL;
  double k = round((double)x * 1.0e6);
  if (k >= 9223372036854775807.0) return 9223372036854775807LL;
  if (k <= -9223372036854775808.0) return (-9223372036854775807LL - 1);
  return (long long)k;
}
RP_HD uint32_t fbits(float x) { union { float f; uint32_t u; } c; c.f = x; return c.u; }
RP_HD uint32_t canon_bits(float x) {
  if (!fin(x)) return 0x7fc00000u;
  uint32_t b = fbits(x);
  return b == 0x80000000u ? 0u : b;
}
RP_HD float signum(float x) { if (isnan(x)) return NAN; return signbit(x) ? -1.0f : 1.0f; }

// float4 <-> f3 / q4
RP_HD f3 xyz(float4 v) { return mk3(v.x, v.y, v.z); }
RP_HD q4 asq(float4 v) { return mkq(v.x, v.y, v.z, v.w); }
RP_HD float4 f4(f3 v, float w = 0.0f) { return make_float4(v.x, v.y, v.z, w); }
RP_HD float4 f4q(q4 q) { return make_float4(q.x, q.y, q.z, q.w); }

}  // namespace rp
