// oracle/oracle_world.cpp -- TEST INFRASTRUCTURE (the oracle). CPU restatement of the
// reference's World::step; see oracle_world.h for scope. Every function cites the reference
// lines it follows (paths relative to the reference's crates/ directory).
#include "oracle_world.h"
#include "oracle_bounce.h"
#include "oracle_joints.h"

#include <algorithm>
#include <climits>
#include <cstring>
#include <cstdio>
#include <numeric>
#include <unordered_map>

#include "blake3_spec.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {
using namespace om;

static const float kMargin = 0.05f;        // MELEE_CCD_MARGIN (step.rs:12)
static const float kPosSlop = 0.005f;      // CONTACT_POS_SLOP (step.rs:16)
static const float kTurnGain = 0.5f;       // TURN_GAIN (step.rs:34)
static const int kTurnMaxSplit = 256;      // TURN_MAX_SPLIT (step.rs:35)
static const float kTurnPrincipal = 1.0e-5f;  // TURN_PRINCIPAL (step.rs:37)
static const float kWarmTol = 0.01f;       // WARM_MATCH_TOL (solver.rs:13)
static const float kCell = 2.5f;           // GridBroadphase::new(2.5) (world.rs:419)

static const Q4 kQId{0, 0, 0, 1};
// Residual histogram bin of an island's last-sweep residual (m/s): <= 1e-4, 1e-3, 1e-2, 1e-1, 1,
// above 1 or NaN (a statistic of this restatement's residual mode; the reference has none).
static uint32_t res_bin(float r) {
  if (r <= 1.0e-4f) return 0u;
  if (r <= 1.0e-3f) return 1u;
  if (r <= 1.0e-2f) return 2u;
  if (r <= 1.0e-1f) return 3u;
  if (r <= 1.0f) return 4u;
  return 5u;
}

// ------------------------------------------------------------------ materials
// props() core table (riftphys-materials/src/materials.rs:97-110), ordinals 0..13.
struct MatProps { float mu_s, mu_k, restitution, stribeck_v; };
static const MatProps kMat[14] = {
    {0.60f, 0.50f, 0.10f, 0.08f},  // Default
    {0.05f, 0.03f, 0.02f, 0.02f},  // Ice
    {1.10f, 0.95f, 0.80f, 0.15f},  // Rubber
    {0.70f, 0.55f, 0.50f, 0.05f},  // Steel
    {1.30f, 1.05f, 0.00f, 0.12f},  // Grit
    {0.55f, 0.45f, 0.08f, 0.10f},  // Wood
    {0.80f, 0.70f, 0.00f, 0.10f},  // Concrete
    {0.90f, 0.80f, 0.00f, 0.12f},  // Asphalt
    {0.80f, 0.60f, 0.20f, 0.10f},  // Leather
    {0.55f, 0.45f, 0.10f, 0.06f},  // Skin
    {1.10f, 0.95f, 0.00f, 0.18f},  // Carpet
    {0.40f, 0.30f, 0.65f, 0.04f},  // Glass
    {0.90f, 0.60f, 0.35f, 0.06f},  // Titanium
    {0.61f, 0.47f, 0.40f, 0.05f},  // Aluminum
};
bool material_known(uint32_t id) { return id < 14; }

// mix_pair + override_for + pair_props (materials.rs:250-305)
PairProps table_pair_props(uint32_t a, uint32_t b) {
  using om::quantize_mat;
  MatProps pa = kMat[a], pb = kMat[b];
  PairProps base;
  base.mu_s = quantize_mat(std::sqrt(std::fabs(pa.mu_s * pb.mu_s)));
  base.mu_k = quantize_mat(std::sqrt(std::fabs(pa.mu_k * pb.mu_k)));
  base.restitution = quantize_mat(rmax(pa.restitution, pb.restitution));
  base.stribeck_v = quantize_mat(0.5f * (pa.stribeck_v + pb.stribeck_v));
  base.stiffness = 0.0f;
  uint32_t x = a < b ? a : b, y = a < b ? b : a;
  // override_for: (Ice, Rubber), (Rubber, Asphalt), (Rubber, Concrete), (Steel, Steel)
  const float* ov = nullptr;
  static const float ice_rubber[4] = {0.20f, 0.10f, 0.05f, 0.08f};
  static const float rubber_asphalt[4] = {1.10f, 0.95f, 0.00f, 0.18f};
  static const float rubber_concrete[4] = {1.00f, 0.85f, 0.00f, 0.16f};
  static const float steel_steel[4] = {0.58f, 0.50f, 0.08f, 0.04f};
  if (x == 1 && y == 2) ov = ice_rubber;
  if (x == 2 && y == 7) ov = rubber_asphalt;
  if (x == 2 && y == 6) ov = rubber_concrete;
  if (x == 3 && y == 3) ov = steel_steel;
  if (ov) {
    base.mu_s = quantize_mat(ov[0]);
    base.mu_k = quantize_mat(ov[1]);
    base.restitution = quantize_mat(ov[2]);
    base.stribeck_v = quantize_mat(ov[3]);
  }
  return base;
}

// ------------------------------------------------------------------ mass properties
// MassProps::finalize / from_*_density (riftphys-geom/src/mass.rs:32-50, 75-145)
static bool valid_pos(float x) { return fin(x) && x > 0.0f; }
static bool finalize_mass(float m, V3 ii, float* inv_mass, V3* inertia) {
  if (!valid_pos(m) || m < 1.0e-12f) { *inv_mass = 0; *inertia = V3{0, 0, 0}; return false; }
  if (!(valid_pos(ii.x) && valid_pos(ii.y) && valid_pos(ii.z))) { *inv_mass = 0; *inertia = V3{0, 0, 0}; return false; }
  *inv_mass = 1.0f / m;
  *inertia = ii;
  return true;
}
bool mass_from_density(uint32_t shape, const float d[3], float rho, float* inv_mass, V3* inertia) {
  const float kPi = 3.14159265358979323846f;
  const float k43 = 4.0f / 3.0f;
  const float k112 = 1.0f / 12.0f;
  if (shape == SH_SPHERE) {
    float r = std::fabs(d[0]);
    if (!(valid_pos(r) && valid_pos(rho))) { *inv_mass = 0; *inertia = V3{0, 0, 0}; return false; }
    float r2 = r * r;
    float vol = ((k43 * kPi) * r2) * r;
    float m = rho * vol;
    float ii = (0.4f * m) * r2;
    return finalize_mass(m, splat(ii), inv_mass, inertia);
  }
  if (shape == SH_BOX) {
    V3 he = vabs(V3{d[0], d[1], d[2]});
    if (!(vfin(he) && valid_pos(rho))) { *inv_mass = 0; *inertia = V3{0, 0, 0}; return false; }
    V3 dims = mul(he, 2.0f);
    if (!(valid_pos(dims.x) && valid_pos(dims.y) && valid_pos(dims.z))) { *inv_mass = 0; *inertia = V3{0, 0, 0}; return false; }
    float vol = (dims.x * dims.y) * dims.z;
    float m = rho * vol;
    float x2 = dims.x * dims.x, y2 = dims.y * dims.y, z2 = dims.z * dims.z;
    float ix = (k112 * m) * (y2 + z2);
    float iy = (k112 * m) * (x2 + z2);
    float iz = (k112 * m) * (x2 + y2);
    return finalize_mass(m, V3{ix, iy, iz}, inv_mass, inertia);
  }
  if (shape == SH_CAPSULE) {
    float r = std::fabs(d[0]), hh = std::fabs(d[1]);
    if (!(valid_pos(r) && fin(rho) && rho > 0.0f)) { *inv_mass = 0; *inertia = V3{0, 0, 0}; return false; }
    float h = hh * 2.0f;
    float r2 = r * r;
    float vol_cyl = (kPi * r2) * h;
    float vol_sph = ((k43 * kPi) * r2) * r;
    float m = rho * (vol_cyl + vol_sph);
    float ix = ((0.25f * m) * r2) + (((k112 * m) * h) * h);
    float iy = (0.5f * m) * r2;
    return finalize_mass(m, V3{ix, iy, ix}, inv_mass, inertia);
  }
  *inv_mass = 0; *inertia = V3{0, 0, 0};
  return false;
}

// ------------------------------------------------------------------ geometry
// Aabb::new (riftphys-geom/src/aabb.rs:21-26): quantise to 1e-6, then order.
static Aabb aabb_new(V3 mn, V3 mx) {
  V3 a{qf32(mn.x), qf32(mn.y), qf32(mn.z)};
  V3 b{qf32(mx.x), qf32(mx.y), qf32(mx.z)};
  return Aabb{vmin(a, b), vmax(a, b)};
}
static Aabb aabb_center_he(V3 c, V3 he) { return aabb_new(sub(c, he), add(c, he)); }
// Aabb::overlaps (aabb.rs:35-39)
static bool overlaps(const Aabb& a, const Aabb& b) {
  return !(a.max.x < b.min.x || a.min.x > b.max.x || a.max.y < b.min.y || a.min.y > b.max.y ||
           a.max.z < b.min.z || a.min.z > b.max.z);
}
// aabb_of (riftphys-geom/src/shape.rs:7-56)
Aabb aabb_of(const Shape& s, const Iso& xf) {
  if (s.kind == SH_SPHERE) {
    return aabb_center_he(xf.pos, splat(std::fabs(s.a)));
  } else if (s.kind == SH_BOX) {
    V3 he{std::fabs(s.a), std::fabs(s.b), std::fabs(s.c)};
    M3 r = mfrom_quat(xf.rot);
    M3 ar{vabs(r.c0), vabs(r.c1), vabs(r.c2)};
    return aabb_center_he(xf.pos, mvec(ar, he));
  } else {  // capsule
    float rr = std::fabs(s.a), h = std::fabs(s.b);
    V3 axis = mul(qrot(xf.rot, V3{0, 1, 0}), h);
    return aabb_center_he(xf.pos, add(vabs(axis), splat(rr)));
  }
}

// ------------------------------------------------------------------ narrowphase
// riftphys-collision/src/narrowphase.rs
static void mpush(Manifold* m, const CP& p) { if (m->len < 4) m->pts[m->len++] = p; }
// norm_or (narrowphase.rs:44-54)
static V3 norm_or(V3 v, V3 fb) {
  v = fin_v(v);
  float l2 = len2(v);
  if (l2 > 1.0e-12f) return mul(v, 1.0f / std::sqrt(l2));
  return fb;
}
static void flip(Manifold* m) {  // flip_manifold (:62-68)
  m->normal = neg(m->normal);
  for (int i = 0; i < m->len; ++i) m->pts[i].normal = m->normal;
}
// reduce_to_4 (:312-338)
static int reduce_to_4(const float* depth, const V3* pt, int n, V3 nrm, int* out) {
  if (n <= 4) { for (int i = 0; i < n; ++i) out[i] = i; return n; }
  auto argmax = [&](auto f, int* bi, float* bv) {
    int best_i = 0; float best_v = -INFINITY; int64_t best_k = INT64_MIN;
    for (int i = 0; i < n; ++i) {
      float v = f(i);
      int64_t k = sort_key6(v);
      if (k > best_k) { best_i = i; best_v = v; best_k = k; }
    }
    *bi = best_i; *bv = best_v;
  };
  int cnt = 0, i0, i1, i2, i3; float v0, d1, a2, a3;
  argmax([&](int i) { return depth[i]; }, &i0, &v0);
  V3 p0 = pt[i0];
  out[cnt++] = i0;
  argmax([&](int i) { return len2(sub(pt[i], p0)); }, &i1, &d1);
  if (!(d1 > 1.0e-12f)) return cnt;
  out[cnt++] = i1;
  V3 e = sub(pt[i1], p0);
  auto side = [&](int i) { return dot(cross(sub(pt[i], p0), e), nrm); };
  argmax([&](int i) { return std::fabs(side(i)); }, &i2, &a2);
  if (!(a2 > 1.0e-12f)) return cnt;
  out[cnt++] = i2;
  float s2 = signum(side(i2));
  argmax([&](int i) { return -side(i) * s2; }, &i3, &a3);
  if (a3 > 1.0e-12f) out[cnt++] = i3;
  return cnt;
}
// clip_poly (:289-301): keeps p.n <= d
static int clip_poly(const V3* in, int n, V3 nn, float d, V3* out) {
  int m = 0;
  for (int i = 0; i < n; ++i) {
    V3 p = in[i], q = in[(i + 1) % n];
    float dp = dot(p, nn) - d, dq = dot(q, nn) - d;
    if (dp <= 0.0f) out[m++] = p;
    if ((dp <= 0.0f) != (dq <= 0.0f)) {
      float t = dp / (dp - dq);
      out[m++] = add(p, mul(sub(q, p), t));
    }
  }
  return m;
}
static float radius3(const V3* ax, const float* e, V3 l) {
  return (e[0] * std::fabs(dot(ax[0], l)) + e[1] * std::fabs(dot(ax[1], l))) + e[2] * std::fabs(dot(ax[2], l));
}
// clip_incident_face (:261-286)
static int clip_incident_face(V3 rc, const float* re, const V3* raxes, int k, V3 nr, V3 ic,
                              const float* ie, const V3* iaxes, V3* poly) {
  int f = 0; float fd = -INFINITY;
  for (int i = 0; i < 3; ++i) { float d = std::fabs(dot(iaxes[i], nr)); if (d > fd) { fd = d; f = i; } }
  float s = dot(iaxes[f], nr) > 0.0f ? -1.0f : 1.0f;
  int u = (f + 1) % 3, v = (f + 2) % 3;
  V3 c = add(ic, mul(iaxes[f], s * ie[f]));
  V3 du = mul(iaxes[u], ie[u]), dv = mul(iaxes[v], ie[v]);
  V3 a[16], b[16];
  a[0] = add(add(c, du), dv); a[1] = add(sub(c, du), dv); a[2] = sub(sub(c, du), dv); a[3] = sub(add(c, du), dv);
  int n = 4;
  int js[2] = {(k + 1) % 3, (k + 2) % 3};
  for (int jj = 0; jj < 2; ++jj) {
    int j = js[jj];
    V3 ax = raxes[j];
    float mid = dot(rc, ax);
    n = clip_poly(a, n, ax, mid + re[j], b);
    if (n == 0) return 0;
    n = clip_poly(b, n, neg(ax), -(mid - re[j]), a);
    if (n == 0) return 0;
  }
  for (int i = 0; i < n; ++i) poly[i] = a[i];
  return n;
}
// collide_box_box (:173-256)
static bool box_box(const Iso& xa, V3 ea, const Iso& xb, V3 eb, float cd, Manifold* m) {
  V3 aa[3] = {qrot(xa.rot, V3{1, 0, 0}), qrot(xa.rot, V3{0, 1, 0}), qrot(xa.rot, V3{0, 0, 1})};
  V3 ba[3] = {qrot(xb.rot, V3{1, 0, 0}), qrot(xb.rot, V3{0, 1, 0}), qrot(xb.rot, V3{0, 0, 1})};
  float ear[3] = {ea.x, ea.y, ea.z}, ebr[3] = {eb.x, eb.y, eb.z};
  V3 t = sub(xb.pos, xa.pos);
  bool have = false; float bo = 0; V3 bl{0, 0, 0}; int bw = 0;
  auto consider = [&](V3 l, int which) -> bool {
    float l2 = len2(l);
    if (l2 < 1.0e-10f) return true;
    l = divs(l, std::sqrt(l2));
    float overlap = (radius3(aa, ear, l) + radius3(ba, ebr, l)) - std::fabs(dot(t, l));
    if (overlap < -cd) return false;
    bool is_face = which < 6;
    bool better;
    if (!have) better = true;
    else {
      bool face = bw < 6;
      if (is_face && face && ((which >= 3) != (bw >= 3))) better = overlap < bo - (0.02f * std::fabs(bo) + 1.0e-3f);
      else if (is_face == face) better = overlap < bo;
      else if (is_face) better = overlap < bo * 1.05f + 1.0e-4f;
      else better = overlap < bo * 0.95f - 1.0e-4f;
    }
    if (better) { have = true; bo = overlap; bl = l; bw = which; }
    return true;
  };
  for (int k = 0; k < 6; ++k) if (!consider(k < 3 ? aa[k] : ba[k - 3], k)) return false;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      if (!consider(cross(aa[i], ba[j]), 6)) return false;
  if (!have) return false;
  V3 n = dot(t, bl) < 0.0f ? neg(bl) : bl;
  V3 normal = norm_or(n, V3{0, 1, 0});
  m->normal = normal; m->len = 0;
  auto edge_point = [&]() {
    V3 sa = add(xa.pos, mul(normal, radius3(aa, ear, normal)));
    V3 sb = sub(xb.pos, mul(normal, radius3(ba, ebr, normal)));
    mpush(m, CP{fin_v(mul(add(sa, sb), 0.5f)), normal, fin0(bo + cd)});
  };
  if (bw == 6) { edge_point(); return true; }
  const Iso* rx; const float* re; const V3* rax; const Iso* ix; const float* ie; const V3* iax; int k; V3 nr;
  if (bw < 3) { rx = &xa; re = ear; rax = aa; ix = &xb; ie = ebr; iax = ba; k = bw; nr = normal; }
  else { rx = &xb; re = ebr; rax = ba; ix = &xa; ie = ear; iax = aa; k = bw - 3; nr = neg(normal); }
  V3 poly[16];
  int np = clip_incident_face(rx->pos, re, rax, k, nr, ix->pos, ie, iax, poly);
  float cdep[16]; V3 cpt[16]; int nc = 0;
  if (np > 0) {
    float plane = dot(rx->pos, nr) + re[k];
    for (int i = 0; i < np; ++i) {
      float depth = plane - dot(poly[i], nr);
      if (depth > -cd) { cdep[nc] = depth; cpt[nc] = add(poly[i], mul(nr, 0.5f * depth)); nc++; }
    }
  }
  if (nc == 0) { edge_point(); return true; }
  int idx[4];
  int r = reduce_to_4(cdep, cpt, nc, normal, idx);
  for (int i = 0; i < r; ++i) mpush(m, CP{fin_v(cpt[idx[i]]), normal, fin0(cdep[idx[i]] + cd)});
  return true;
}
// collide_sphere_sphere (:412-442)
static bool sphere_sphere(V3 ca, float ra, V3 cb, float rb, float cd, Manifold* m) {
  V3 delta = sub(cb, ca);
  float d2 = len2(delta);
  ra = fin0(rmax(ra, 0.0f)); rb = fin0(rmax(rb, 0.0f));
  float allowed = fin0((ra + rb) + cd);
  if (!fin(d2) || d2 > allowed * allowed) return false;
  float dist = std::sqrt(d2);
  V3 raw = dist > 1.0e-6f ? divs(delta, dist) : V3{1, 0, 0};
  V3 normal = norm_or(raw, V3{1, 0, 0});
  float pen = fin0(rmax(allowed - dist, 0.0f));
  V3 pa = add(ca, mul(normal, ra)), pb = sub(cb, mul(normal, rb));
  m->normal = normal; m->len = 0;
  mpush(m, CP{fin_v(mul(add(pa, pb), 0.5f)), normal, pen});
  return true;
}
static void capsule_segment(const Iso& xf, float half, V3* a, V3* b) {  // :445-449
  V3 axis = qrot(xf.rot, V3{0, 1, 0});
  float h = std::fabs(half);
  *a = sub(xf.pos, mul(axis, h));
  *b = add(xf.pos, mul(axis, h));
}
static V3 closest_point_segment(V3 p, V3 a, V3 b) {  // :452-460
  V3 ab = sub(b, a);
  float l2 = len2(ab);
  if (l2 <= 1.0e-12f) return a;
  float t = clampf(dot(sub(p, a), ab) / l2, 0.0f, 1.0f);
  return add(a, mul(ab, t));
}
static void closest_seg_seg(V3 p0, V3 p1, V3 q0, V3 q1, V3* pa, V3* pb) {  // :462-509
  V3 u = sub(p1, p0), v = sub(q1, q0), w = sub(p0, q0);
  float a = dot(u, u), b = dot(u, v), c = dot(v, v), d = dot(u, w), e = dot(v, w);
  float d0 = a * c - b * b;
  float sn, tn, sd = d0, td = d0;
  const float EPS = 1.0e-6f;
  if (d0 < EPS) { sn = 0.0f; sd = 1.0f; tn = e; td = c; }
  else {
    sn = b * e - c * d;
    tn = a * e - b * d;
    if (sn < 0.0f) { sn = 0.0f; tn = e; td = c; }
    else if (sn > sd) { sn = sd; tn = e + b; td = c; }
  }
  if (tn < 0.0f) {
    tn = 0.0f;
    if (-d < 0.0f) sn = 0.0f;
    else if (-d > a) sn = sd;
    else { sn = -d; sd = a; }
  } else if (tn > td) {
    tn = td;
    if ((-d + b) < 0.0f) sn = 0.0f;
    else if ((-d + b) > a) sn = sd;
    else { sn = -d + b; sd = a; }
  }
  float sc = std::fabs(sn) < EPS ? 0.0f : sn / sd;
  float tc = std::fabs(tn) < EPS ? 0.0f : tn / td;
  *pa = add(p0, mul(u, sc));
  *pb = add(q0, mul(v, tc));
}
static bool capsule_sphere(const Iso& cx, float cr, float ch, V3 sc, float sr, float cd, Manifold* m) {
  V3 a, b; capsule_segment(cx, ch, &a, &b);
  return sphere_sphere(closest_point_segment(sc, a, b), cr, sc, sr, cd, m);
}
static bool capsule_capsule(const Iso& xa, float ra, float ha, const Iso& xb, float rb, float hb, float cd, Manifold* m) {
  V3 a0, a1, b0, b1; capsule_segment(xa, ha, &a0, &a1); capsule_segment(xb, hb, &b0, &b1);
  V3 pa, pb; closest_seg_seg(a0, a1, b0, b1, &pa, &pb);
  return sphere_sphere(pa, ra, pb, rb, cd, m);
}
// collide_box_sphere (:540-593)
static bool box_sphere(const Iso& bx, V3 e, V3 sc, float sr, float cd, Manifold* m) {
  V3 pl = fin_v(qrot(qconj(bx.rot), sub(sc, bx.pos)));
  V3 cl{rmin(rmax(pl.x, -e.x), e.x), rmin(rmax(pl.y, -e.y), e.y), rmin(rmax(pl.z, -e.z), e.z)};
  float r = fin0(rmax(sr, 0.0f));
  float allowed = fin0(r + cd);
  V3 yw = qrot(bx.rot, V3{0, 1, 0});
  if (veq(cl, pl)) {
    V3 dtf = sub(e, vabs(pl));
    V3 axis; float depth;
    if (dtf.x < dtf.y && dtf.x < dtf.z) { axis = mul(V3{1, 0, 0}, pl.x > 0.0f ? 1.0f : -1.0f); depth = dtf.x; }
    else if (dtf.y < dtf.z) { axis = mul(V3{0, 1, 0}, pl.y > 0.0f ? 1.0f : -1.0f); depth = dtf.y; }
    else { axis = mul(V3{0, 0, 1}, pl.z > 0.0f ? 1.0f : -1.0f); depth = dtf.z; }
    V3 normal = norm_or(qrot(bx.rot, axis), yw);
    V3 face = fin_v(add(sc, mul(normal, depth)));
    float pen = fin0(allowed + rmax(depth, 0.0f));
    V3 position = fin_v(mul(add(face, sub(sc, mul(normal, r))), 0.5f));
    m->normal = normal; m->len = 0;
    mpush(m, CP{position, normal, pen});
    return true;
  }
  V3 cw = fin_v(add(bx.pos, qrot(bx.rot, cl)));
  V3 delta = sub(sc, cw);
  float dist = std::sqrt(len2(delta));
  if (dist > allowed) return false;
  V3 raw = dist > 1.0e-6f ? divs(delta, dist) : yw;
  V3 normal = norm_or(raw, yw);
  float pen = fin0(allowed - dist);
  V3 position = fin_v(mul(add(cw, sub(sc, mul(normal, r))), 0.5f));
  m->normal = normal; m->len = 0;
  mpush(m, CP{position, normal, pen});
  return true;
}
// collide_box_capsule (:595-622)
static bool box_capsule(const Iso& bx, V3 e, const Iso& cx, float cr, float ch, float cd, Manifold* m) {
  V3 aw, bw; capsule_segment(cx, ch, &aw, &bw);
  Q4 inv = qconj(bx.rot);
  V3 al = fin_v(qrot(inv, sub(aw, bx.pos)));
  V3 bl = fin_v(qrot(inv, sub(bw, bx.pos)));
  V3 mid = closest_point_segment(V3{0, 0, 0}, al, bl);
  V3 tp[3] = {al, bl, mid};
  bool have = false;
  for (int i = 0; i < 3; ++i) {
    V3 pw = add(bx.pos, qrot(bx.rot, tp[i]));
    Manifold t;
    if (box_sphere(bx, e, pw, cr, cd, &t)) {
      if (!have || t.pts[0].penetration > m->pts[0].penetration) { *m = t; have = true; }
    }
  }
  return have;
}
// closest_point_triangle (:627-669)
static V3 closest_point_triangle(V3 p, V3 a, V3 b, V3 c) {
  V3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  float d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) return a;
  V3 bp = sub(p, b);
  float d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) return b;
  float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) { float v = d1 / (d1 - d3); return add(a, mul(ab, v)); }
  V3 cp = sub(p, c);
  float d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) return c;
  float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) { float w = d2 / (d2 - d6); return add(a, mul(ac, w)); }
  float va = d3 * d6 - d5 * d4;
  if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
    float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return add(b, mul(sub(c, b), w));
  }
  float denom = 1.0f / ((va + vb) + vc);
  float v = vb * denom, w = vc * denom;
  return add(add(a, mul(ab, v)), mul(ac, w));
}
static void tri_world(const Shape& t, V3* a, V3* b, V3* c) {  // tri_xf = IDENTITY
  V3 z{0, 0, 0};
  *a = add(z, qrot(kQId, t.ta)); *b = add(z, qrot(kQId, t.tb)); *c = add(z, qrot(kQId, t.tc));
}
// collide_sphere_triangle (:671-707)
static bool sphere_triangle(V3 sc, float sr, const Shape& tri, float cd, Manifold* m) {
  V3 a, b, c; tri_world(tri, &a, &b, &c);
  V3 cl = closest_point_triangle(sc, a, b, c);
  V3 delta = sub(sc, cl);
  float d2 = len2(delta);
  float r = fin0(rmax(sr, 0.0f));
  float allowed = fin0(r + cd);
  if (d2 > allowed * allowed) return false;
  float dist = std::sqrt(d2);
  V3 tn = normalize_or_zero(cross(sub(b, a), sub(c, a)));
  V3 raw = dist > 1.0e-6f ? divs(delta, dist) : tn;
  V3 normal = norm_or(raw, tn);
  m->normal = normal; m->len = 0;
  mpush(m, CP{fin_v(cl), normal, fin0(allowed - dist)});
  return true;
}
// collide_capsule_triangle (:709-733)
static bool capsule_triangle(const Iso& cx, float cr, float ch, const Shape& tri, float cd, Manifold* m) {
  V3 aw, bw; capsule_segment(cx, ch, &aw, &bw);
  V3 mid = mul(add(aw, bw), 0.5f);
  V3 tp[3] = {aw, bw, mid};
  bool have = false;
  for (int i = 0; i < 3; ++i) {
    Manifold t;
    if (sphere_triangle(tp[i], cr, tri, cd, &t)) {
      if (!have || t.pts[0].penetration > m->pts[0].penetration) { *m = t; have = true; }
    }
  }
  return have;
}
// collide_box_triangle (:349-409)
static bool box_triangle(const Iso& bx, V3 e, const Shape& tri, float cd, Manifold* m) {
  V3 ta, tb, tc; tri_world(tri, &ta, &tb, &tc);
  V3 raw = cross(sub(tb, ta), sub(tc, ta));
  if (!(len2(raw) > 1.0e-12f) || !vfin(raw)) return false;
  V3 n = normalize(raw);
  V3 ax[3] = {qrot(bx.rot, V3{1, 0, 0}), qrot(bx.rot, V3{0, 1, 0}), qrot(bx.rot, V3{0, 0, 1})};
  float er[3] = {e.x, e.y, e.z};
  float r = radius3(ax, er, n);
  float centre = dot(sub(bx.pos, ta), n);
  if (centre - r > cd) return false;
  int f = 0; float fd = -INFINITY;
  for (int i = 0; i < 3; ++i) { float d = std::fabs(dot(ax[i], n)); if (d > fd) { fd = d; f = i; } }
  float sgn = dot(ax[f], n) > 0.0f ? -1.0f : 1.0f;
  int u = (f + 1) % 3, v = (f + 2) % 3;
  V3 c = add(bx.pos, mul(ax[f], sgn * er[f]));
  V3 du = mul(ax[u], er[u]), dv = mul(ax[v], er[v]);
  V3 pa[16], pb[16];
  pa[0] = add(add(c, du), dv); pa[1] = add(sub(c, du), dv); pa[2] = sub(sub(c, du), dv); pa[3] = sub(add(c, du), dv);
  int np = 4;
  V3 ep[3][2] = {{ta, tb}, {tb, tc}, {tc, ta}};
  for (int k = 0; k < 3; ++k) {
    V3 p = ep[k][0], q = ep[k][1];
    V3 out = cross(sub(q, p), n);
    if (!(len2(out) > 1.0e-12f)) return false;
    out = normalize(out);
    np = clip_poly(pa, np, out, dot(p, out), pb);
    if (np == 0) return false;
    for (int i = 0; i < np; ++i) pa[i] = pb[i];
  }
  float cdep[16]; V3 cpt[16]; int nc = 0;
  for (int i = 0; i < np; ++i) {
    float dist = dot(sub(pa[i], ta), n);
    if (dist <= cd) { cdep[nc] = -dist; cpt[nc] = sub(pa[i], mul(n, 0.5f * dist)); nc++; }
  }
  if (nc == 0) return false;
  V3 normal = neg(n);
  m->normal = normal; m->len = 0;
  int idx[4];
  int rr = reduce_to_4(cdep, cpt, nc, normal, idx);
  for (int i = 0; i < rr; ++i) mpush(m, CP{fin_v(cpt[idx[i]]), normal, fin0(cd + cdep[idx[i]])});
  return true;
}
// collide_shapes (:73-161)
bool collide_shapes(const Shape& a, const Iso& xa, const Shape& b, const Iso& xb, float cd, Manifold* m) {
  if (!vfin(xa.pos) || !vfin(xb.pos)) return false;
  cd = fin0(rmax(cd, 0.0f));
  uint32_t ka = a.kind, kb = b.kind;
  bool ok = false;
  if (ka == SH_SPHERE && kb == SH_SPHERE) ok = sphere_sphere(xa.pos, a.a, xb.pos, b.a, cd, m);
  else if (ka == SH_CAPSULE && kb == SH_SPHERE) ok = capsule_sphere(xa, a.a, a.b, xb.pos, b.a, cd, m);
  else if (ka == SH_SPHERE && kb == SH_CAPSULE) { ok = capsule_sphere(xb, b.a, b.b, xa.pos, a.a, cd, m); if (ok) flip(m); }
  else if (ka == SH_CAPSULE && kb == SH_CAPSULE) ok = capsule_capsule(xa, a.a, a.b, xb, b.a, b.b, cd, m);
  else if (ka == SH_BOX && kb == SH_SPHERE) ok = box_sphere(xa, V3{a.a, a.b, a.c}, xb.pos, b.a, cd, m);
  else if (ka == SH_SPHERE && kb == SH_BOX) { ok = box_sphere(xb, V3{b.a, b.b, b.c}, xa.pos, a.a, cd, m); if (ok) flip(m); }
  else if (ka == SH_BOX && kb == SH_CAPSULE) ok = box_capsule(xa, V3{a.a, a.b, a.c}, xb, b.a, b.b, cd, m);
  else if (ka == SH_CAPSULE && kb == SH_BOX) { ok = box_capsule(xb, V3{b.a, b.b, b.c}, xa, a.a, a.b, cd, m); if (ok) flip(m); }
  else if (ka == SH_BOX && kb == SH_BOX) ok = box_box(xa, V3{a.a, a.b, a.c}, xb, V3{b.a, b.b, b.c}, cd, m);
  else if (ka == SH_SPHERE && kb == SH_TRIANGLE) ok = sphere_triangle(xa.pos, a.a, b, cd, m);
  else if (ka == SH_CAPSULE && kb == SH_TRIANGLE) ok = capsule_triangle(xa, a.a, a.b, b, cd, m);
  else if (ka == SH_BOX && kb == SH_TRIANGLE) ok = box_triangle(xa, V3{a.a, a.b, a.c}, b, cd, m);
  return ok;
}

// ------------------------------------------------------------------ world
World::World(uint32_t capacity) {
  awake.assign(capacity, 1);
  sleep_ticks.assign(capacity, 0);
  sleep_allowed.assign(capacity, 1);
  alive.assign(capacity, 0);
}

// Bodies::inv_inertia_world (dynamics.rs:158-163)
M3 World::inv_inertia_world(uint32_t i) const {
  if (inv_mass[i] == 0.0f) return mzero();
  M3 r = mfrom_quat(rot[i]);
  return mmul(mmul(r, inv_I[i]), mtranspose(r));
}
// fin_q (dynamics.rs:15-20)
static Q4 fin_q(Q4 q) {
  if (!qfin(q)) return kQId;
  Q4 qq = qnormalize(q);
  if (!qfin(qq)) return kQId;
  if (qq.w < 0.0f) qq = qneg(qq);
  return qq;
}
// Bodies::set_pose / set_vel (dynamics.rs:130-145)
void World::set_pose(uint32_t i, const Iso& p) {
  if (vfin(p.pos)) pos[i] = fin_v(p.pos);
  if (qfin(p.rot)) rot[i] = fin_q(p.rot);
}
void World::set_vel(uint32_t i, V3 l, V3 a) {
  if (vfin(l)) lin[i] = fin_v(l);
  if (vfin(a)) ang[i] = fin_v(a);
}
// Bodies::apply_impulse / apply_angular_impulse (dynamics.rs:193-205)
void World::apply_impulse(uint32_t i, V3 j) {
  float im = inv_mass[i];
  if (im > 0.0f && vfin(j)) lin[i] = fin_v(add(lin[i], mul(j, im)));
}
void World::apply_angular_impulse(uint32_t i, V3 tau) {
  if (inv_mass[i] > 0.0f && vfin(tau)) {
    V3 dw = mvec(inv_inertia_world(i), tau);
    ang[i] = fin_v(add(ang[i], dw));
  }
}
// World::add_body (world.rs:595-614) + Bodies::add (dynamics.rs:98-117)
uint32_t World::add_body(const Iso& pose, V3 l, V3 a, float inv_mass_in, V3 inertia_diag, bool dynamic) {
  float im_arg = dynamic ? inv_mass_in : 0.0f;
  M3 inertia = mdiag(inertia_diag);
  float det = mdet(inertia);
  bool has_inv = dynamic && fin(det) && det > 0.0f;
  M3 inv_local = has_inv ? minverse(inertia) : mzero();
  bool is_dyn = dynamic && fin(im_arg) && im_arg > 0.0f;
  float im = is_dyn ? fin0(im_arg) : 0.0f;
  pos.push_back(vfin(pose.pos) ? pose.pos : V3{0, 0, 0});
  rot.push_back(fin_q(pose.rot));
  lin.push_back(vfin(l) ? l : V3{0, 0, 0});
  ang.push_back(vfin(a) ? a : V3{0, 0, 0});
  inv_mass.push_back(im);
  dyn.push_back(is_dyn ? 1 : 0);
  bool inv_fin = vfin(inv_local.c0) && vfin(inv_local.c1) && vfin(inv_local.c2);
  M3 ii = !is_dyn ? mzero() : (has_inv && inv_fin ? inv_local : mdiag(splat(im)));
  inv_I.push_back(ii);
  uint32_t id = (uint32_t)pos.size() - 1;
  if (last_lin_vel.size() <= id) last_lin_vel.resize(id + 1, V3{0, 0, 0});
  last_lin_vel[id] = l;
  if (id >= awake.size()) { awake.resize(id + 1, 1); sleep_ticks.resize(id + 1, 0); sleep_allowed.resize(id + 1, 1); }
  wake(id);
  if (alive.size() <= id) alive.resize(id + 1, 0);
  alive[id] = 1;
  return id;
}
// World::add_collider (world.rs:616-622)
void World::add_collider(uint32_t body, const Shape& s, uint32_t mat) {
  Collider c{body, s, aabb_of(s, Iso{pos[body], rot[body]}), mat};
  colliders.push_back(c);
}
void World::wake(uint32_t id) { awake[id] = 1; sleep_ticks[id] = 0; }  // sleep.rs:22-26
// World::drop_warm_of (world.rs:818-833)
void World::drop_warm_of(uint32_t b) {
  for (auto it = warm.begin(); it != warm.end();) {
    if (std::get<0>(it->first) == b || std::get<1>(it->first) == b) it = warm.erase(it); else ++it;
  }
  for (auto it = warm_joints.begin(); it != warm_joints.end();) {
    const Joint& j = joints[it->first];
    if (j.a == b || j.b == b) it = warm_joints.erase(it); else ++it;
  }
}
// World::set_body_pose (world.rs:501-513)
void World::set_body_pose(uint32_t id, const Iso& p) {
  drop_warm_of(id);
  set_pose(id, p);
  for (auto& c : colliders) if (c.body == id) c.aabb = aabb_of(c.shape, p);
}
// World::set_body_vel (world.rs:674-687)
void World::set_body_vel(uint32_t id, V3 l, V3 a) {
  set_vel(id, l, a);
  if (id < last_lin_vel.size()) last_lin_vel[id] = l;
}
// World::apply_impulse (world.rs:689-692)
void World::apply_impulse_world(uint32_t id, V3 j) { wake(id); apply_impulse(id, j); }
// World::remove_body (world.rs:696-713) + Bodies::deactivate (dynamics.rs:213-220)
bool World::remove_body(uint32_t id) {
  if (id >= pos.size() || !alive[id]) return false;
  alive[id] = 0;
  lin[id] = V3{0, 0, 0}; ang[id] = V3{0, 0, 0};
  inv_mass[id] = 0.0f; dyn[id] = 0; inv_I[id] = mzero();
  colliders.erase(std::remove_if(colliders.begin(), colliders.end(), [&](const Collider& c) { return c.body == id; }), colliders.end());
  drop_warm_of(id);
  return true;
}
// World::pair_props (world.rs:982-986)
PairProps World::pair_props(uint32_t a, uint32_t b) const {
  std::pair<uint32_t, uint32_t> key = a <= b ? std::make_pair(a, b) : std::make_pair(b, a);
  for (auto& o : overrides) if (o.first == key) return o.second;
  return table_pair_props(a, b);
}
void World::set_pair_props(uint32_t a, uint32_t b, const PairProps& p) {  // world.rs:975-979
  std::pair<uint32_t, uint32_t> key = a <= b ? std::make_pair(a, b) : std::make_pair(b, a);
  overrides.erase(std::remove_if(overrides.begin(), overrides.end(), [&](auto& o) { return o.first == key; }), overrides.end());
  overrides.push_back({key, p});
}
void World::update_colliders_aabb() {  // world.rs:793-798
  for (auto& c : colliders) c.aabb = aabb_of(c.shape, Iso{pos[c.body], rot[c.body]});
}
uint32_t World::num_sleeping() const {
  uint32_t n = 0;
  for (auto a : awake) n += a == 0;
  return n;
}
CarriedState World::carried_state() const {  // world.rs:912-923
  CarriedState s;
  s.warm = warm; s.warm_joints = warm_joints; s.last_lin_vel = last_lin_vel; s.awake = awake; s.sleep_ticks = sleep_ticks;
  return s;
}
void World::restore_carried_state(const CarriedState& s) {  // world.rs:927-961
  warm = s.warm;
  for (size_t i = 0; i < s.last_lin_vel.size() && i < last_lin_vel.size(); ++i) last_lin_vel[i] = s.last_lin_vel[i];
  for (size_t i = 0; i < s.awake.size() && i < s.sleep_ticks.size(); ++i) {
    if (i < awake.size()) { awake[i] = s.awake[i]; sleep_ticks[i] = s.sleep_ticks[i]; }
  }
  auto al = [&](uint32_t b) { return b == 0xFFFFFFFFu || (b < alive.size() && alive[b] != 0); };
  for (auto it = warm.begin(); it != warm.end();) {
    if (!(al(std::get<0>(it->first)) && al(std::get<1>(it->first)))) it = warm.erase(it); else ++it;
  }
  warm_joints = s.warm_joints;
  for (auto it = warm_joints.begin(); it != warm_joints.end();) {
    bool keep = it->first < joints.size() && al(joints[it->first].a) && al(joints[it->first].b);
    if (!keep) it = warm_joints.erase(it); else ++it;
  }
}

// ------------------------------------------------------------------ broadphase
// GridBroadphase::run (riftphys-collision/src/broadphase.rs:29-99)
static void broadphase(const std::vector<Aabb>& ab, std::vector<std::pair<uint32_t, uint32_t>>& pairs) {
  struct KH { size_t operator()(const std::tuple<int, int, int>& k) const {
    return ((size_t)(uint32_t)std::get<0>(k) * 73856093u) ^ ((size_t)(uint32_t)std::get<1>(k) * 19349663u) ^ ((size_t)(uint32_t)std::get<2>(k) * 83492791u);
  } };
  std::unordered_map<std::tuple<int, int, int>, std::vector<uint32_t>, KH> grid;
  std::vector<uint32_t> oversized;
  pairs.clear();
  auto cell = [](float v) -> int {  // (v / cell).floor() as i32, saturating, NaN -> 0
    float f = std::floor(v / kCell);
    if (std::isnan(f)) return 0;
    if (f >= 2147483647.0f) return 2147483647;
    if (f <= -2147483648.0f) return INT32_MIN;
    return (int)f;
  };
  for (uint32_t i = 0; i < ab.size(); ++i) {
    const Aabb& a = ab[i];
    if (!fin(a.min.x)) continue;
    float dx = a.max.x - a.min.x, dy = a.max.y - a.min.y, dz = a.max.z - a.min.z;
    if (dx > kCell * 5.0f || dy > kCell * 5.0f || dz > kCell * 5.0f) { oversized.push_back(i); continue; }
    int x0 = cell(a.min.x), x1 = cell(a.max.x), y0 = cell(a.min.y), y1 = cell(a.max.y), z0 = cell(a.min.z), z1 = cell(a.max.z);
    for (long x = x0; x <= x1; ++x)
      for (long y = y0; y <= y1; ++y)
        for (long z = z0; z <= z1; ++z) grid[std::make_tuple((int)x, (int)y, (int)z)].push_back(i);
  }
  for (auto& kv : grid) {
    auto& c = kv.second;
    for (size_t i = 0; i < c.size(); ++i)
      for (size_t j = i + 1; j < c.size(); ++j) {
        uint32_t a = c[i], b = c[j];
        uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
        if (overlaps(ab[lo], ab[hi])) pairs.push_back({lo, hi});
      }
  }
  for (uint32_t big : oversized)
    for (uint32_t i = 0; i < ab.size(); ++i)
      if (i != big && overlaps(ab[big], ab[i])) pairs.push_back(i < big ? std::make_pair(i, big) : std::make_pair(big, i));
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
}

// HeightField::query_aabb (riftphys-terrain/src/terrain.rs:300-358)
static void hf_query(const HeightField& hf, const Aabb& a, std::vector<Shape>& out) {
  int nx = (int)hf.nx, nz = (int)hf.nz;
  if (nx < 2 || nz < 2) return;
  auto toi = [](float f) -> long {
    if (std::isnan(f)) return 0;
    if (f >= 2147483647.0f) return 2147483647;
    if (f <= -2147483648.0f) return INT32_MIN;
    return (long)f;
  };
  auto cl = [](long v, long lo, long hi) { return v < lo ? lo : (v > hi ? hi : v); };
  float lminx = a.min.x - hf.ox, lmaxx = a.max.x - hf.ox, lminz = a.min.z - hf.oz, lmaxz = a.max.z - hf.oz;
  long gx0 = cl((long)(int32_t)toi(std::floor(lminx / hf.sx)) - 1, 0, nx - 2);
  long gx1 = cl((long)(int32_t)toi(std::ceil(lmaxx / hf.sx)) + 1, 0, nx - 2);
  long gz0 = cl((long)(int32_t)toi(std::floor(lminz / hf.sz)) - 1, 0, nz - 2);
  long gz1 = cl((long)(int32_t)toi(std::ceil(lmaxz / hf.sz)) + 1, 0, nz - 2);
  if (a.min.y > hf.max_y + 1.0f || a.max.y < hf.min_y - 1.0f) return;
  for (long gz = gz0; gz <= gz1; ++gz)
    for (long gx = gx0; gx <= gx1; ++gx) {
      auto H = [&](long x, long z) { return hf.h[(size_t)x + (size_t)z * hf.nx]; };
      float h00 = H(gx, gz), h10 = H(gx + 1, gz), h01 = H(gx, gz + 1), h11 = H(gx + 1, gz + 1);
      float x0 = (float)gx * hf.sx + hf.ox, x1 = x0 + hf.sx;
      float z0 = (float)gz * hf.sz + hf.oz, z1 = z0 + hf.sz;
      V3 p00{x0, h00, z0}, p10{x1, h10, z0}, p01{x0, h01, z1}, p11{x1, h11, z1};
      Shape t1{SH_TRIANGLE, 0, 0, 0, p00, p01, p10};
      Shape t2{SH_TRIANGLE, 0, 0, 0, p10, p01, p11};
      out.push_back(t1);
      out.push_back(t2);
    }
}

// ------------------------------------------------------------------ queries
// normal_from_aabb_point / ray_aabb (riftphys-world/src/world/geom.rs:40-93)
static V3 normal_from_aabb_point(const Aabb& b, V3 p) {
  const float eps = 1.0e-4f;
  if (std::fabs(p.x - b.min.x) < eps) return V3{-1, 0, 0};
  if (std::fabs(p.x - b.max.x) < eps) return V3{1, 0, 0};
  if (std::fabs(p.y - b.min.y) < eps) return V3{0, -1, 0};
  if (std::fabs(p.y - b.max.y) < eps) return V3{0, 1, 0};
  if (std::fabs(p.z - b.min.z) < eps) return V3{0, 0, -1};
  if (std::fabs(p.z - b.max.z) < eps) return V3{0, 0, 1};
  V3 c = mul(add(b.min, b.max), 0.5f);
  V3 n = sub(p, c);
  float l2 = dot(n, n);
  if (l2 > 1.0e-20f) n = divs(n, std::sqrt(l2));
  else n = V3{0, 1, 0};
  return n;
}
static bool ray_aabb(V3 o, V3 d, const Aabb& b, float max_d, float* t_out, V3* p_out, V3* n_out) {
  const float eps = 1.0e-8f;
  float tmin = 0.0f, tmax = max_d;
  const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z};
  const float lo[3] = {b.min.x, b.min.y, b.min.z}, hi[3] = {b.max.x, b.max.y, b.max.z};
  for (int a = 0; a < 3; ++a) {
    if (std::fabs(dd[a]) < eps) {
      if (oo[a] < lo[a] || oo[a] > hi[a]) return false;
    } else {
      float inv = 1.0f / dd[a];
      float t1 = (lo[a] - oo[a]) * inv, t2 = (hi[a] - oo[a]) * inv;
      if (t1 > t2) std::swap(t1, t2);
      if (t1 > tmin) tmin = t1;
      if (t2 < tmax) tmax = t2;
      if (tmin > tmax) return false;
    }
  }
  if (tmin < 0.0f || tmin > max_d) return false;
  V3 p = add(o, mul(d, tmin));
  *t_out = tmin;
  *p_out = p;
  *n_out = normal_from_aabb_point(b, p);
  return true;
}
// Triangle::intersect_ray (riftphys-geom/src/triangle.rs:215-235) with Plane::from_points /
// from_point_normal / intersect_ray (plane.rs:16-86) and Triangle::barycentric (triangle.rs:74-113)
static bool ray_triangle(V3 o, V3 d, float max_d, V3 a, V3 b, V3 c, float* t_out) {
  V3 n = cross(sub(b, a), sub(c, a));
  float a2 = dot(n, n);
  if (!fin(a2) || a2 <= 1.0e-16f) return false;
  if (!(vfin(a) && vfin(b) && vfin(c))) return false;
  float l2 = dot(n, n);
  if (!fin(l2) || l2 <= 1.0e-6f * 1.0e-6f) return false;
  float inv_len = 1.0f / std::sqrt(l2);
  V3 nu = mul(n, inv_len);
  float pd = -dot(nu, a);
  if (!(vfin(nu) && fin(pd))) return false;
  if (!(vfin(o) && vfin(d))) return false;
  float denom = dot(nu, d);
  if (!fin(denom) || std::fabs(denom) < 1.0e-6f) return false;
  float numer = -(dot(nu, o) + pd);
  if (!fin(numer)) return false;
  float t = numer / denom;
  if (!fin(t)) return false;
  if (!(t >= 0.0f && t <= max_d)) return false;
  V3 p = add(o, mul(d, t));
  V3 v0 = sub(b, a), v1 = sub(c, a), v2 = sub(p, a);
  float d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
  float den = d00 * d11 - d01 * d01;
  float scale = rmax(std::fabs(d00 * d11), 1.0f);
  if (!fin(den) || std::fabs(den) <= 1.0e-12f * scale) return false;
  float inv = 1.0f / den;
  float v = (d11 * d20 - d01 * d21) * inv;
  float w = (d00 * d21 - d01 * d20) * inv;
  float u = 1.0f - v - w;
  if (!(fin(u) && fin(v) && fin(w) && u >= -1.0e-5f && v >= -1.0e-5f && w >= -1.0e-5f)) return false;
  *t_out = t;
  return true;
}
// Triangle::normal (triangle.rs:26-31)
static V3 tri_normal(V3 a, V3 b, V3 c) {
  V3 n = cross(sub(b, a), sub(c, a));
  if (!vfin(n)) return V3{0, 0, 0};
  float rcp = 1.0f / std::sqrt(dot(n, n));
  return (fin(rcp) && rcp > 0.0f) ? mul(n, rcp) : V3{0, 0, 0};
}
bool World::raycast(V3 origin, V3 dir, float max_dist, uint32_t ignore, uint32_t* body, float* toi, V3* point,
                    V3* normal) const {
  const float max_d = rmax(max_dist, 0.0f);
  if (max_d <= 0.0f) return false;
  const float l = std::sqrt(dot(dir, dir));
  if (!fin(l) || l < 1.0e-12f) return false;
  dir = divs(dir, l);
  bool have = false;
  float bt = 0.0f;
  size_t bci = 0;
  V3 bp{0, 0, 0}, bn{0, 0, 0};
  const size_t kEnv = (size_t)-1;
  for (size_t ci = 0; ci < colliders.size(); ++ci) {
    const Collider& c = colliders[ci];
    if (c.body == ignore) continue;
    float t;
    V3 p, n;
    if (!ray_aabb(origin, dir, c.aabb, max_d, &t, &p, &n)) continue;
    if (!have || (t < bt - 1.0e-9f) || (std::fabs(t - bt) <= 1.0e-9f && ci < bci)) {
      have = true; bt = t; bci = ci; bp = p; bn = n;
    }
  }
  if (has_hf) {
    V3 end = add(origin, mul(dir, max_d));
    Aabb q = aabb_new(vmin(origin, end), vmax(origin, end));
    std::vector<Shape> tris;
    hf_query(hf, q, tris);
    for (const Shape& tr : tris) {
      float t;
      if (!ray_triangle(origin, dir, max_d, tr.ta, tr.tb, tr.tc, &t)) continue;
      if (!have || t < bt - 1.0e-9f) {
        have = true; bt = t; bci = kEnv;
        bp = fin(t) ? add(origin, mul(dir, t)) : origin;
        bn = tri_normal(tr.ta, tr.tb, tr.tc);
      }
    }
  }
  if (!have) return false;
  *body = bci == kEnv ? 0xFFFFFFFFu : colliders[bci].body;
  *toi = clampf(bt / max_d, 0.0f, 1.0f);
  *point = bp;
  *normal = bn;
  return true;
}

// ---- exact ray casts: ray_shape (riftphys-geom/src/raycast.rs:13-130) against true shapes
static bool ray_sphere_local(V3 o, V3 d, V3 c, float r, float* t_out, V3* n_out) {  // raycast.rs:42-53
  const V3 m = sub(o, c);
  const float b = dot(m, d);
  const float cc = dot(m, m) - r * r;
  if (cc <= 0.0f) { *t_out = 0.0f; *n_out = neg(d); return true; }
  if (b > 0.0f) return false;
  const float disc = b * b - cc;
  if (disc < 0.0f) return false;
  float t = -b - std::sqrt(disc);
  t = rmax(t, 0.0f);
  *t_out = t;
  *n_out = normalize_or_zero(add(m, mul(d, t)));
  return true;
}
static bool ray_box_local(V3 o, V3 d, V3 he, float* t_out, V3* n_out) {  // raycast.rs:55-82
  float tmin = 0.0f, tmax = INFINITY;
  V3 normal = neg(d);
  const float oa[3] = {o.x, o.y, o.z}, da[3] = {d.x, d.y, d.z}, ha[3] = {he.x, he.y, he.z};
  for (int ax = 0; ax < 3; ++ax) {
    if (std::fabs(da[ax]) < 1.0e-9f) {
      if (oa[ax] < -ha[ax] || oa[ax] > ha[ax]) return false;
      continue;
    }
    const float inv = 1.0f / da[ax];
    float t1 = (-ha[ax] - oa[ax]) * inv, t2 = (ha[ax] - oa[ax]) * inv;
    float sign = -1.0f;
    if (t1 > t2) { std::swap(t1, t2); sign = 1.0f; }
    if (t1 > tmin) {
      tmin = t1;
      float n[3] = {0.0f, 0.0f, 0.0f};
      n[ax] = sign;
      normal = V3{n[0], n[1], n[2]};
    }
    tmax = rmin(tmax, t2);
    if (tmin > tmax) return false;
  }
  *t_out = tmin;
  *n_out = normal;
  return true;
}
static bool ray_tube_local(V3 o, V3 d, float r, float hh, float* t_out, V3* n_out) {  // raycast.rs:84-96
  const float a = d.x * d.x + d.z * d.z;
  if (a < 1.0e-9f) return false;
  const float b = o.x * d.x + o.z * d.z;
  const float c = o.x * o.x + o.z * o.z - r * r;
  const float disc = b * b - a * c;
  if (disc < 0.0f) return false;
  const float t = (-b - std::sqrt(disc)) / a;
  if (t < 0.0f) return false;
  const V3 p = add(o, mul(d, t));
  if (std::fabs(p.y) > hh) return false;
  *t_out = t;
  *n_out = normalize_or_zero(V3{p.x, 0.0f, p.z});
  return true;
}
static bool ray_capsule_local(V3 o, V3 d, float r, float hh, float* t_out, V3* n_out) {  // raycast.rs:98-109
  const V3 core{0.0f, clampf(o.y, -hh, hh), 0.0f};
  const V3 oc = sub(o, core);
  if (dot(oc, oc) <= r * r) { *t_out = 0.0f; *n_out = neg(d); return true; }
  bool have = ray_tube_local(o, d, r, hh, t_out, n_out);
  const float cys[2] = {hh, -hh};
  for (float cy : cys) {
    float t;
    V3 n;
    if (ray_sphere_local(o, d, V3{0.0f, cy, 0.0f}, r, &t, &n) && (!have || t < *t_out)) {
      have = true; *t_out = t; *n_out = n;
    }
  }
  return have;
}
// ray_shape for the colliders' shapes and terrain triangles: (t, world normal facing the ray)
static bool ray_shape(const Shape& s, const Iso& xf, V3 origin, V3 dir, float max_t, float* t_out, V3* n_out) {
  if (!(max_t >= 0.0f) || !vfin(origin) || !vfin(dir)) return false;
  const Q4 inv = qconj(xf.rot);
  const V3 o = qrot(inv, sub(origin, xf.pos));
  const V3 d = qrot(inv, dir);
  float t;
  V3 n;
  bool hit;
  if (s.kind == SH_SPHERE) hit = ray_sphere_local(o, d, V3{0, 0, 0}, std::fabs(s.a), &t, &n);
  else if (s.kind == SH_BOX) hit = ray_box_local(o, d, V3{std::fabs(s.a), std::fabs(s.b), std::fabs(s.c)}, &t, &n);
  else if (s.kind == SH_CAPSULE) hit = ray_capsule_local(o, d, std::fabs(s.a), std::fabs(s.b), &t, &n);
  else {  // a triangle (triangle.rs:215-235 and :26-31)
    hit = ray_triangle(o, d, max_t, s.ta, s.tb, s.tc, &t);
    if (hit) {
      const V3 tn = tri_normal(s.ta, s.tb, s.tc);
      n = dot(tn, d) > 0.0f ? neg(tn) : tn;
    }
  }
  if (!hit || !(t <= max_t && fin(t))) return false;
  *t_out = t;
  *n_out = qrot(xf.rot, n);
  return true;
}
// World::raycast_exact (queries.rs:18-48), skipping one body index (0xFFFFFFFF: none): colliders
// whose fresh AABB the ray meets, then the terrain triangles in the ray's box; a hit replaces the
// best only when strictly nearer.
bool World::raycast_exact(V3 origin, V3 dir, float max_dist, uint32_t ignore, uint32_t* body, float* toi, V3* point,
                          V3* normal) const {
  const float max_d = rmax(max_dist, 0.0f);
  if (max_d <= 0.0f) return false;
  const float l = std::sqrt(dot(dir, dir));
  if (!fin(l) || l < 1.0e-12f) return false;
  dir = divs(dir, l);
  bool have = false;
  float bt = 0.0f;
  size_t bci = 0;
  V3 bn{0, 0, 0};
  const size_t kEnv = (size_t)-1;
  for (size_t ci = 0; ci < colliders.size(); ++ci) {
    const Collider& c = colliders[ci];
    if (c.body == ignore) continue;
    const Iso pose{pos[c.body], rot[c.body]};
    float t0;
    V3 p0, n0;
    if (!ray_aabb(origin, dir, aabb_of(c.shape, pose), max_d, &t0, &p0, &n0)) continue;
    float t;
    V3 n;
    if (ray_shape(c.shape, pose, origin, dir, max_d, &t, &n) && (!have || t < bt)) {
      have = true; bt = t; bci = ci; bn = n;
    }
  }
  if (has_hf) {
    const V3 end = add(origin, mul(dir, max_d));
    const Aabb q = aabb_new(vmin(origin, end), vmax(origin, end));
    std::vector<Shape> tris;
    hf_query(hf, q, tris);
    const Iso id{V3{0, 0, 0}, Q4{0, 0, 0, 1}};
    for (const Shape& tr : tris) {
      float t;
      V3 n;
      if (ray_shape(tr, id, origin, dir, max_d, &t, &n) && (!have || t < bt)) {
        have = true; bt = t; bci = kEnv; bn = n;
      }
    }
  }
  if (!have) return false;
  *body = bci == kEnv ? 0xFFFFFFFFu : colliders[bci].body;
  *toi = clampf(bt / max_d, 0.0f, 1.0f);
  *point = add(origin, mul(dir, bt));
  *normal = bn;
  return true;
}

// ---- capsule sweeps: riftphys-query/src/lib.rs:1-134 (sphere sweeps against AABBs)
static const float kToiEps = 1e-9f;
static bool ray_aabb_slab_unit(V3 o, V3 d, const Aabb& b, float* t_out, V3* n_out) {  // lib.rs:42-79
  V3 inv{(o.x == o.x && std::fabs(d.x) > 1e-9f) ? 1.0f / d.x : 1.0e9f,
         (o.y == o.y && std::fabs(d.y) > 1e-9f) ? 1.0f / d.y : 1.0e9f,
         (o.z == o.z && std::fabs(d.z) > 1e-9f) ? 1.0f / d.z : 1.0e9f};
  V3 t1{(b.min.x - o.x) * inv.x, (b.min.y - o.y) * inv.y, (b.min.z - o.z) * inv.z};
  V3 t2{(b.max.x - o.x) * inv.x, (b.max.y - o.y) * inv.y, (b.max.z - o.z) * inv.z};
  V3 tmin = vmin(t1, t2), tmax = vmax(t1, t2);
  float t_enter = tmin.x;
  V3 n{t1.x > t2.x ? 1.0f : -1.0f, 0.0f, 0.0f};
  if (tmin.y > t_enter) { t_enter = tmin.y; n = V3{0.0f, t1.y > t2.y ? 1.0f : -1.0f, 0.0f}; }
  if (tmin.z > t_enter) { t_enter = tmin.z; n = V3{0.0f, 0.0f, t1.z > t2.z ? 1.0f : -1.0f}; }
  float t_exit = rmin(rmin(tmax.x, tmax.y), tmax.z);
  if (t_enter <= t_exit && t_exit >= 0.0f && t_enter >= 0.0f && t_enter <= 1.0f) { *t_out = t_enter; *n_out = n; return true; }
  return false;
}
static bool sweep_sphere_aabb(V3 p0, V3 v, float r, const Aabb& a, float* t, V3* n) {  // lib.rs:81-104, dt 1
  V3 dir = mul(v, 1.0f);
  Aabb e{sub(a.min, splat(r)), add(a.max, splat(r))};
  if (dot(dir, dir) < 1e-12f) {
    bool inside = p0.x >= e.min.x && p0.x <= e.max.x && p0.y >= e.min.y && p0.y <= e.max.y && p0.z >= e.min.z && p0.z <= e.max.z;
    if (inside) { *t = 0.0f; *n = V3{0, 1, 0}; }
    return inside;
  }
  return ray_aabb_slab_unit(p0, dir, e, t, n);
}
// sweep_two_spheres_aabbs over one AABB (lib.rs:118-134) with pick_better (lib.rs:14-33)
static bool sweep_two(V3 tip0, V3 base0, V3 v, float r, const Aabb& a, float* t, V3* n, int* kind) {
  bool have = false;
  float tt;
  V3 nn;
  if (sweep_sphere_aabb(tip0, v, r, a, &tt, &nn)) { have = true; *t = tt; *n = nn; *kind = 0; }
  if (sweep_sphere_aabb(base0, v, r, a, &tt, &nn)) {
    if (!have || tt < *t - kToiEps) { have = true; *t = tt; *n = nn; *kind = 1; }
  }
  return have;
}
bool World::sweep_capsule(V3 from, V3 to, float radius, float half_height, uint32_t ignore, uint32_t* body,
                          float* toi, bool* overlap, V3* point, V3* normal) const {
  const V3 v = sub(to, from);
  const float dist_sq = dot(v, v);
  const Shape cap{SH_CAPSULE, radius, half_height, 0.0f, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}};
  const Iso cx{from, Q4{0, 0, 0, 1}};
  *overlap = false;
  for (size_t ci = 0; ci < colliders.size(); ++ci) {  // 1. overlap at t = 0
    const Collider& c = colliders[ci];
    if (c.body == ignore) continue;
    Manifold m;
    if (collide_shapes(cap, cx, c.shape, Iso{pos[c.body], rot[c.body]}, 0.0f, &m) && m.len > 0) {
      *body = c.body; *toi = 0.0f; *overlap = true; *point = m.pts[0].position; *normal = m.normal;
      return true;
    }
  }
  std::vector<Shape> tris;
  if (has_hf) {
    hf_query(hf, aabb_of(cap, cx), tris);
    for (const Shape& tr : tris) {
      Manifold m;
      if (collide_shapes(cap, cx, tr, Iso{V3{0, 0, 0}, Q4{0, 0, 0, 1}}, 0.0f, &m) && m.len > 0) {
        *body = 0xFFFFFFFFu; *toi = 0.0f; *overlap = true; *point = m.pts[0].position; *normal = m.normal;
        return true;
      }
    }
  }
  if (dist_sq < 1.0e-12f) return false;  // 2. stationary
  const V3 tip0 = add(from, V3{0.0f, half_height, 0.0f}), base0 = add(from, V3{0.0f, -half_height, 0.0f});
  bool have = false;
  float bt = 0.0f;
  size_t bci = 0;
  const size_t kEnv = (size_t)-1;
  V3 bp{0, 0, 0}, bn{0, 0, 0};
  for (size_t ci = 0; ci < colliders.size(); ++ci) {  // 3. swept spheres against AABBs
    const Collider& c = colliders[ci];
    if (c.body == ignore) continue;
    float t;
    V3 n;
    int kind;
    if (!sweep_two(tip0, base0, v, radius, c.aabb, &t, &n, &kind)) continue;
    t = clampf(t, 0.0f, 1.0f);
    V3 c0 = kind == 0 ? tip0 : base0;
    V3 p = sub(add(c0, mul(v, t)), mul(n, radius));
    if (!have || (t < bt - kToiEps) || (std::fabs(t - bt) <= kToiEps && ci < bci)) { have = true; bt = t; bci = ci; bp = p; bn = n; }
  }
  if (has_hf) {
    V3 ext = splat(radius + half_height);
    Aabb sb = aabb_new(sub(vmin(from, to), ext), add(vmax(from, to), ext));
    tris.clear();
    hf_query(hf, sb, tris);
    const Q4 id{0, 0, 0, 1};
    for (const Shape& tr : tris) {
      V3 wa = add(V3{0, 0, 0}, qrot(id, tr.ta)), wb = add(V3{0, 0, 0}, qrot(id, tr.tb)), wc = add(V3{0, 0, 0}, qrot(id, tr.tc));
      Aabb ea = aabb_new(vmin(vmin(wa, wb), wc), vmax(vmax(wa, wb), wc));
      float t;
      V3 n;
      int kind;
      if (!sweep_two(tip0, base0, v, radius, ea, &t, &n, &kind)) continue;
      t = clampf(t, 0.0f, 1.0f);
      V3 c0 = kind == 0 ? tip0 : base0;
      V3 p = sub(add(c0, mul(v, t)), mul(n, radius));
      if (!have || t < bt - kToiEps) { have = true; bt = t; bci = kEnv; bp = p; bn = n; }
    }
  }
  if (!have) return false;
  *body = bci == kEnv ? 0xFFFFFFFFu : colliders[bci].body;
  *toi = bt;
  *point = bp;
  *normal = bn;
  return true;
}

// ---- the kinematic player controller
uint32_t World::add_player(const Iso& pose) {
  uint32_t id = add_body(pose, V3{0, 0, 0}, V3{0, 0, 0}, 0.0f, V3{0, 0, 0}, false);
  Player p;
  p.body = id;
  add_collider(id, Shape{SH_CAPSULE, p.radius, p.height * 0.5f, 0.0f, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}}, 0);
  players.push_back(p);
  return (uint32_t)players.size() - 1;
}
static bool aabb_intersects(const Aabb& a, const Aabb& b) {  // Aabb::intersects (aabb.rs:75-79)
  return a.min.x <= b.max.x && a.max.x >= b.min.x && a.min.y <= b.max.y && a.max.y >= b.min.y && a.min.z <= b.max.z &&
         a.max.z >= b.min.z;
}
// World::update_players (step.rs:544-639): gravity or the sticky floor, the input direction at the
// player's speed, then up to four sweep-and-slide passes: the first terrain triangle, else the first
// collider, within 5 cm of the moved capsule pushes it out and kills the motion into it (a floor
// grounds it; a dynamic body is woken and kicked). Poses move through Bodies::set_pose, so the
// colliders' stored AABBs stay those of the step's start until the tick updates them.
void World::update_players(float dt) {
  for (size_t pi = 0; pi < players.size(); ++pi) {
    Player pl = players[pi];
    V3 p = pos[pl.body];
    if (!pl.grounded) pl.vertical_vel -= 9.81f * dt;
    else if (pl.vertical_vel <= 0.0f) pl.vertical_vel = -0.5f;
    const float im2 = dot(pl.input, pl.input);
    V3 move_dir = im2 > 1e-6f ? divs(pl.input, std::sqrt(im2)) : V3{0, 0, 0};
    V3 desired = add(mul(mul(move_dir, pl.speed), dt), V3{0.0f, pl.vertical_vel * dt, 0.0f});
    pl.grounded = false;
    for (int it = 0; it < 4; ++it) {
      if (dot(desired, desired) < 1e-6f) break;
      const Iso xf{add(p, desired), Q4{0, 0, 0, 1}};
      const Shape sh{SH_CAPSULE, pl.radius, pl.height * 0.5f, 0.0f, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}};
      const Aabb box = aabb_of(sh, xf);
      bool have = false;
      V3 hn{0, 0, 0};
      float hpen = 0.0f;
      long hbody = -1;
      if (has_hf) {
        std::vector<Shape> tris;
        hf_query(hf, box, tris);
        for (const Shape& tr : tris) {
          Manifold m{};
          if (collide_shapes(sh, xf, tr, Iso{V3{0, 0, 0}, Q4{0, 0, 0, 1}}, 0.05f, &m)) {
            have = true; hn = m.pts[0].normal; hpen = m.pts[0].penetration;
            break;
          }
        }
      }
      if (!have) {
        for (const Collider& c : colliders) {
          if (c.body == pl.body || !aabb_intersects(box, c.aabb)) continue;
          Manifold m{};
          if (collide_shapes(sh, xf, c.shape, Iso{pos[c.body], rot[c.body]}, 0.05f, &m)) {
            have = true; hn = m.pts[0].normal; hpen = m.pts[0].penetration; hbody = (long)c.body;
            break;
          }
        }
      }
      if (!have) break;
      if (hn.y > 0.6f) { pl.grounded = true; pl.vertical_vel = 0.0f; }
      desired = add(desired, mul(hn, hpen + 0.001f));
      const float d = dot(desired, hn);
      if (d < 0.0f) desired = sub(desired, mul(hn, d));
      if (hbody >= 0 && dyn[(size_t)hbody]) {
        wake((uint32_t)hbody);
        apply_impulse((uint32_t)hbody, mul(neg(hn), 10.0f));
      }
    }
    p = add(p, desired);
    set_pose(pl.body, Iso{p, Q4{0, 0, 0, 1}});
    players[pi] = pl;
  }
}

// ------------------------------------------------------------------ solver
// ContactConstraint (solver.rs:47-87), the fields the configured path reads.
struct CC {
  uint32_t ai, bi;
  bool terrain;
  float inv_a, inv_b;
  M3 ii_a, ii_b;
  V3 ra, rb;
  float m_n, m_t1, m_t2;
  V3 n, t1, t2;
  float mu_s, mu_k, sv;
  float depth_bias, restitution_bias;
  bool soft, toi;
  // W6 (solver.rs:575-587): the gap at the step's start, the pair's restitution, and each side's
  // normal velocity at the contact from the start velocities and after this step's forces
  float toi_s0, toi_e, toi_va0, toi_va1, toi_vb0, toi_vb1;
};
// orthonormal_basis (riftphys-world/src/world/geom.rs:30-38)
static void orthonormal_basis(V3 n, V3* t1, V3* t2) {
  float ax = std::fabs(n.x), ay = std::fabs(n.y), az = std::fabs(n.z);
  V3 base = (ax <= ay && ax <= az) ? V3{1, 0, 0} : (ay <= az ? V3{0, 1, 0} : V3{0, 0, 1});
  *t1 = normalize_or_zero(cross(base, n));
  *t2 = cross(n, *t1);
}
static float mu_dynamic(const CC& cs, float slip) {  // solver.rs:429-431
  float t = slip / cs.sv;
  return cs.mu_k + (cs.mu_s - cs.mu_k) * expf_rp(-(t * t));
}
static V3 contact_rel_vel(const World& w, const CC& cs) {  // solver.rs:443-451
  V3 va = add(w.lin[cs.ai], cross(w.ang[cs.ai], cs.ra));
  V3 vb = cs.terrain ? V3{0, 0, 0} : add(w.lin[cs.bi], cross(w.ang[cs.bi], cs.rb));
  return sub(vb, va);
}
static float slip_speed(const World& w, const CC& cs) {  // solver.rs:435-439
  V3 v = contact_rel_vel(w, cs);
  float a = dot(v, cs.t1), b = dot(v, cs.t2);
  return std::sqrt(a * a + b * b);
}
static void apply_contact_impulse(World& w, const CC& cs, V3 j) {  // solver.rs:455-464
  if (cs.inv_a > 0.0f) { V3 nj = neg(j); w.apply_impulse(cs.ai, nj); w.apply_angular_impulse(cs.ai, cross(cs.ra, nj)); }
  if (cs.inv_b > 0.0f) { w.apply_impulse(cs.bi, j); w.apply_angular_impulse(cs.bi, cross(cs.rb, j)); }
}
static float eff_mass(float ia, float ib, const M3& IA, const M3& IB, V3 ra, V3 rb, V3 d) {
  V3 ca = cross(ra, d), cb = cross(rb, d);
  float k = ((ia + ib) + dot(ca, mvec(IA, ca))) + dot(cb, mvec(IB, cb));
  return k > 1.0e-9f ? 1.0f / k : 0.0f;
}
// The level schedule of solver.rs:621-642 over an order of rows; returns levels per row
// (0xFFFFFFFF for rows with no writable body).
static uint32_t level_schedule(const std::vector<CC>& cs, const std::vector<uint32_t>& order, uint32_t nb,
                               std::vector<uint32_t>& level, std::vector<std::vector<uint32_t>>& batches) {
  std::vector<uint32_t> bl(nb, 0);
  level.assign(cs.size(), 0xFFFFFFFFu);
  batches.clear();
  for (uint32_t ci : order) {
    const CC& c = cs[ci];
    bool wa = c.inv_a > 0.0f, wb = !c.terrain && c.inv_b > 0.0f;
    if (!wa && !wb) continue;
    uint32_t la = wa ? bl[c.ai] : 0, lb = wb ? bl[c.bi] : 0;
    uint32_t t = la > lb ? la : lb;
    if (t >= batches.size()) batches.emplace_back();
    batches[t].push_back(ci);
    level[ci] = t;
    if (wa) bl[c.ai] = t + 1;
    if (wb) bl[c.bi] = t + 1;
  }
  return (uint32_t)batches.size();
}

// ------------------------------------------------------------------ the tick
// ------------------------------------------------------------------ W6 bounce passes
// toi_bounce (solver.rs:203-219): the end-of-step normal velocity of a bounce found at its time of
// impact inside the step and, when the pair started apart, the pseudo-velocity that moves it to
// where the bounce leaves it.
static void toi_bounce(float s0, float v0, float a, float e, float dt, float* v_end_out, bool* has_pseudo, float* pseudo) {
  float t_c;
  if (s0 <= 0.0f) {
    t_c = 0.0f;
  } else {
    float disc = v0 * v0 - 2.0f * a * s0;
    float den = disc >= 0.0f ? -v0 + std::sqrt(disc) : 0.0f;
    t_c = den > 0.0f ? rmin(2.0f * s0 / den, dt) : dt;
  }
  float v_out = rmax(-e * (v0 + a * t_c), 0.0f);
  float tau = dt - t_c;
  float rise = v_out * tau + 0.5f * a * tau * tau;
  float v_end, s_end;
  if (rise < 0.0f) { v_end = 0.0f; s_end = 0.0f; }
  else { v_end = rmax(v_out + a * tau, 0.0f); s_end = rise; }
  *v_end_out = v_end;
  *has_pseudo = s0 > 0.0f;
  *pseudo = (s_end - s0) / dt - v_end;
}
// row_sides (solver.rs:117-134): a side that cannot move (no inverse mass, zero inverse inertia)
// is none; the world inverse inertia symmetrised in f64.
static std::array<bounce::RowSide, 2> row_sides(const CC& cs) {
  using namespace bounce;
  const D3 n{cs.n.x, cs.n.y, cs.n.z};
  auto side = [&](uint32_t body, double sign, V3 r, float inv, const M3& ii) {
    RowSide s{};
    if (inv <= 0.0f && mis_zero(ii)) { s.body = kNone; return s; }
    s.body = body;
    s.jl = dmul(n, sign);
    s.ja = dmul(dcross(D3{r.x, r.y, r.z}, n), sign);
    auto c = [](V3 v) { return D3{v.x, v.y, v.z}; };
    DM3 m{c(ii.c0), c(ii.c1), c(ii.c2)};
    DM3 mt{D3{m.c0.x, m.c1.x, m.c2.x}, D3{m.c0.y, m.c1.y, m.c2.y}, D3{m.c0.z, m.c1.z, m.c2.z}};
    DM3 ms{dmul(dadd(m.c0, mt.c0), 0.5), dmul(dadd(m.c1, mt.c1), 0.5), dmul(dadd(m.c2, mt.c2), 0.5)};
    s.mjl = dmul(s.jl, (double)inv);
    s.mja = dmvec(ms, s.ja);
    return s;
  };
  return {side(cs.ai, -1.0, cs.ra, cs.inv_a, cs.ii_a), side(cs.terrain ? kNone : cs.bi, 1.0, cs.rb, cs.inv_b, cs.ii_b)};
}
// The W6 bounce passes (solver.rs:1009-1241) for free bodies' contacts approaching faster than
// 1 m/s with restitution: each bounces at its time of impact (its end-of-step velocity target from
// toi_bounce), with the bounced bodies' other loaded contacts as push-only supports, solved per
// connected component by the interior-point LCP (up to 250 rows) or swept; then the pseudo pass
// moves the bounced pairs to where the bounce leaves them (pseudo-velocities for the integration).
static constexpr size_t kDirectMax = 250, kBounceSweeps = 256, kBounceSolves = 64;
static constexpr float kBounceTol = 1e-6f;
static void w6_bounce(World& w, const std::vector<CC>& cons, std::vector<float>& acc_jn, const std::vector<float>& acc_jt,
                      const std::vector<uint8_t>& jointed, float dt, uint32_t num_bodies,
                      std::vector<std::pair<V3, V3>>& pseudo_out, uint32_t* n_toi) {
  using namespace bounce;
  const size_t nc = cons.size();
  auto loaded_at = [&](size_t c, const std::vector<float>& jn) {
    return jn[c] > 0.0f || acc_jt[2 * c] != 0.0f || acc_jt[2 * c + 1] != 0.0f;
  };
  auto grow = [&](std::vector<uint8_t>& involved, const std::vector<float>& jn) {
    for (;;) {
      bool changed = false;
      for (size_t c = 0; c < nc; ++c) {
        const CC& cs = cons[c];
        if (cs.soft || cs.terrain || !loaded_at(c, jn)) continue;
        const uint32_t xs[2] = {cs.ai, cs.bi}, ys[2] = {cs.bi, cs.ai};
        const float invy[2] = {cs.inv_b, cs.inv_a};
        for (int k = 0; k < 2; ++k)
          if (involved[xs[k]] && !involved[ys[k]] && invy[k] > 0.0f && !jointed[ys[k]]) {
            involved[ys[k]] = 1;
            changed = true;
          }
      }
      if (!changed) break;
    }
  };
  auto partner = [&](const CC& cs, uint32_t id) { return cs.terrain ? 0xFFFFFFFFu : (id == cs.ai ? cs.bi : cs.ai); };
  // cs with jointed bodies immovable and its normal effective mass; false if neither side moves
  auto free_only = [&](const CC& in, CC* out) {
    CC cs = in;
    if (jointed[cs.ai]) { cs.inv_a = 0.0f; cs.ii_a = mzero(); }
    if (cs.terrain || jointed[cs.bi]) { cs.inv_b = 0.0f; cs.ii_b = mzero(); }
    V3 ca = cross(cs.ra, cs.n), cb = cross(cs.rb, cs.n);
    float k = ((cs.inv_a + cs.inv_b) + dot(ca, mvec(cs.ii_a, ca))) + dot(cb, mvec(cs.ii_b, cb));
    if (!(k > 1e-9f)) return false;
    cs.m_n = 1.0f / k;
    *out = cs;
    return true;
  };
  std::vector<uint8_t> toi_set(nc, 0);
  bool any = false;
  for (size_t c = 0; c < nc; ++c) {
    toi_set[c] = cons[c].toi && cons[c].restitution_bias > 0.0f && acc_jn[c] > 0.0f;
    any = any || toi_set[c];
  }
  std::vector<std::pair<size_t, float>> toi_rows, pseudo_rows;
  if (any) {
    std::vector<std::vector<uint32_t>> rests_on(num_bodies);
    for (size_t c = 0; c < nc; ++c) {
      const CC& cs = cons[c];
      if (toi_set[c] || !loaded_at(c, acc_jn)) continue;
      rests_on[cs.ai].push_back(partner(cs, cs.ai));
      if (!cs.terrain) rests_on[cs.bi].push_back(partner(cs, cs.bi));
    }
    for (size_t c = 0; c < nc; ++c) {
      if (!toi_set[c]) continue;
      const CC& cs = cons[c];
      // a side resting on something other than its partner is struck from its start velocity
      auto side = [&](uint32_t id, float start, float after, float* s0, float* s1) {
        uint32_t other = partner(cs, id);
        bool rests = false;
        for (uint32_t p : rests_on[id]) rests = rests || p != other;
        *s0 = start;
        *s1 = rests ? start : after;
      };
      float a0, a1, b0 = 0.0f, b1 = 0.0f;
      side(cs.ai, cs.toi_va0, cs.toi_va1, &a0, &a1);
      if (!cs.terrain) side(cs.bi, cs.toi_vb0, cs.toi_vb1, &b0, &b1);
      float v0 = b0 - a0;
      float acc = ((b1 - a1) - v0) / dt;
      float v_end, u;
      bool hp;
      toi_bounce(cs.toi_s0, v0, acc, cs.toi_e, dt, &v_end, &hp, &u);
      toi_rows.push_back({c, v_end});
      if (hp) pseudo_rows.push_back({c, u});
    }
    std::vector<uint8_t> involved(num_bodies, 0);
    for (auto& tr : toi_rows) {
      const CC& cs = cons[tr.first];
      involved[cs.ai] = 1;
      if (!cs.terrain) involved[cs.bi] = 1;
    }
    grow(involved, acc_jn);
    // one list: the bounces (accumulating into acc_jn), then the supports (fresh accumulators)
    struct BRow { CC cs; float target; long c; };
    std::vector<BRow> rows;
    for (auto& tr : toi_rows) rows.push_back(BRow{cons[tr.first], tr.second, (long)tr.first});
    for (size_t c = 0; c < nc; ++c) {
      const CC& cs = cons[c];
      if (toi_set[c] || cs.soft || acc_jn[c] <= 0.0f) continue;
      if (!involved[cs.ai] && (cs.terrain || !involved[cs.bi])) continue;
      CC row;
      if (!free_only(cs, &row)) continue;
      rows.push_back(BRow{row, rmin(cs.depth_bias, 0.0f), -1});
    }
    std::vector<float> sup_acc(rows.size(), 0.0f);
    std::vector<std::array<RowSide, 2>> sides_all;
    for (auto& r : rows) sides_all.push_back(row_sides(r.cs));
    for (auto& comp : row_components(sides_all, num_bodies)) {
      const size_t n = comp.size();
      bool sweep = n > kDirectMax;
      auto acc_of = [&](size_t i) -> float& { return rows[i].c >= 0 ? acc_jn[(size_t)rows[i].c] : sup_acc[i]; };
      if (!sweep) {
        std::vector<std::array<RowSide, 2>> sides;
        for (size_t i : comp) sides.push_back(sides_all[i]);
        Csr k = contact_csr(sides);
        std::vector<double> b, acc0;
        for (size_t i : comp) {
          b.push_back((double)(rows[i].target - dot(contact_rel_vel(w, rows[i].cs), rows[i].cs.n)));
          acc0.push_back((double)acc_of(i));
        }
        QpResult qr = bounce_qp(k, b, acc0, kBounceSolves);
        sweep = !qr.converged;
        for (size_t q = 0; q < n; ++q) {
          size_t i = comp[q];
          float old = acc_of(i);
          float nw = rmax((float)((double)old + qr.x[q]), 0.0f);
          acc_of(i) = nw;
          apply_contact_impulse(w, rows[i].cs, mul(rows[i].cs.n, nw - old));
        }
      }
      if (!sweep) continue;
      for (size_t it = 0; it < kBounceSweeps; ++it) {
        float change = 0.0f;
        for (size_t m = 0; m < n; ++m) {
          size_t i = comp[it % 2 == 0 ? m : n - 1 - m];
          const CC& row = rows[i].cs;
          float v = dot(contact_rel_vel(w, row), row.n);
          float old = acc_of(i);
          float nw = rmax(old + (rows[i].target - v) * row.m_n, 0.0f);
          acc_of(i) = nw;
          apply_contact_impulse(w, row, mul(row.n, nw - old));
          change = rmax(change, std::fabs(nw - old) / row.m_n / (1.0f + std::fabs(rows[i].target)));
        }
        if (change < kBounceTol) break;
      }
    }
  }
  *n_toi = (uint32_t)toi_rows.size();
  // 3c. the pseudo pass (:1161-1241)
  if (pseudo_rows.empty()) return;
  std::vector<uint8_t> in_set(nc, 0), involved(num_bodies, 0);
  for (auto& pr : pseudo_rows) {
    in_set[pr.first] = 1;
    const CC& cs = cons[pr.first];
    involved[cs.ai] = 1;
    if (!cs.terrain) involved[cs.bi] = 1;
  }
  grow(involved, acc_jn);
  std::vector<std::pair<CC, float>> rows;
  for (auto& pr : pseudo_rows) {
    CC row;
    if (free_only(cons[pr.first], &row)) rows.push_back({row, pr.second});
  }
  for (size_t c = 0; c < nc; ++c) {
    const CC& cs = cons[c];
    if (in_set[c] || cs.soft || !loaded_at(c, acc_jn)) continue;
    if (!involved[cs.ai] && (cs.terrain || !involved[cs.bi])) continue;
    CC row;
    if (free_only(cs, &row)) rows.push_back({row, 0.0f});
  }
  std::vector<std::pair<V3, V3>> pseudo(num_bodies, {V3{0, 0, 0}, V3{0, 0, 0}});
  auto rel = [&](const CC& cs) {
    V3 la = pseudo[cs.ai].first, wa = pseudo[cs.ai].second;
    V3 lb = cs.terrain ? V3{0, 0, 0} : pseudo[cs.bi].first, wb = cs.terrain ? V3{0, 0, 0} : pseudo[cs.bi].second;
    return dot(sub(add(lb, cross(wb, cs.rb)), add(la, cross(wa, cs.ra))), cs.n);
  };
  std::vector<std::array<RowSide, 2>> sides_all;
  for (auto& r : rows) sides_all.push_back(row_sides(r.first));
  std::vector<std::pair<D3, D3>> acc(num_bodies, {D3{0, 0, 0}, D3{0, 0, 0}});
  std::vector<uint8_t> direct(num_bodies, 0);
  for (auto& comp : row_components(sides_all, num_bodies)) {
    const size_t n = comp.size();
    if (n <= kDirectMax) {
      std::vector<std::array<RowSide, 2>> sides;
      for (size_t i : comp) sides.push_back(sides_all[i]);
      Csr k = contact_csr(sides);
      std::vector<double> u;
      for (size_t i : comp) u.push_back((double)rows[i].second);
      std::vector<double> x = pseudo_solve(k, u);
      for (size_t q = 0; q < n; ++q)
        for (auto& sd : sides[q]) {
          if (sd.body == kNone) continue;
          acc[sd.body].first = dadd(acc[sd.body].first, dmul(sd.mjl, x[q]));
          acc[sd.body].second = dadd(acc[sd.body].second, dmul(sd.mja, x[q]));
          direct[sd.body] = 1;
        }
      continue;
    }
    for (size_t it = 0; it < kBounceSweeps; ++it) {
      float change = 0.0f;
      for (size_t m = 0; m < n; ++m) {
        const CC& cs = rows[comp[it % 2 == 0 ? m : n - 1 - m]].first;
        float u = rows[comp[it % 2 == 0 ? m : n - 1 - m]].second;
        float d = u - rel(cs);
        change = rmax(change, std::fabs(d) / (1.0f + std::fabs(u)));
        V3 j = mul(cs.n, d * cs.m_n);
        if (cs.inv_a > 0.0f) {
          pseudo[cs.ai].first = sub(pseudo[cs.ai].first, mul(j, cs.inv_a));
          pseudo[cs.ai].second = sub(pseudo[cs.ai].second, mvec(cs.ii_a, cross(cs.ra, j)));
        }
        if (cs.inv_b > 0.0f) {
          pseudo[cs.bi].first = add(pseudo[cs.bi].first, mul(j, cs.inv_b));
          pseudo[cs.bi].second = add(pseudo[cs.bi].second, mvec(cs.ii_b, cross(cs.rb, j)));
        }
      }
      if (change < kBounceTol) break;
    }
  }
  for (uint32_t b = 0; b < num_bodies; ++b)
    if (direct[b]) {
      const D3 l = acc[b].first, a = acc[b].second;
      pseudo[b] = {V3{(float)l.x, (float)l.y, (float)l.z}, V3{(float)a.x, (float)a.y, (float)a.z}};
    }
  pseudo_out = std::move(pseudo);
}

void World::step(float dt) {
  const uint32_t count = num_bodies();
  tick += 1;
  stats = Stats{};
  update_players(dt);  // step.rs:51
  // --- Stage 1: forces (step.rs:53-68)
  std::vector<V3> pre_lin(lin.begin(), lin.end()), pre_ang(ang.begin(), ang.end());
  V3 g{q6(gravity.x), q6(gravity.y), q6(gravity.z)};  // grav_eval Uniform (gravity.rs:79-87)
  for (uint32_t i = 0; i < count; ++i) {
    if (!dyn[i] || !awake[i]) continue;
    V3 l = add(lin[i], mul(g, dt));
    set_vel(i, l, ang[i]);
  }
  // --- Stage 2: broadphase (step.rs:70-83)
  update_colliders_aabb();
  const uint32_t ncol = (uint32_t)colliders.size();
  std::vector<float> sweep(ncol);
  std::vector<Aabb> swept(ncol);
  for (uint32_t c = 0; c < ncol; ++c) {
    const Collider& co = colliders[c];
    float reach = 0.5f * len(sub(co.aabb.max, co.aabb.min));  // Collider::reach (world.rs:97-100)
    sweep[c] = kMargin + (len(lin[co.body]) + len(ang[co.body]) * reach) * dt;
    swept[c] = Aabb{sub(co.aabb.min, splat(sweep[c])), add(co.aabb.max, splat(sweep[c]))};
  }
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  broadphase(swept, pairs);
  stats.pairs = (uint32_t)pairs.size();
  last_pairs = pairs;
  // --- Stage 2: narrowphase (step.rs:85-142); bodies joined by a joint do not collide
  std::vector<uint64_t> jointed_pairs;
  for (auto& jt : joints) {
    uint32_t lo = std::min(jt.a, jt.b), hi = std::max(jt.a, jt.b);
    jointed_pairs.push_back(((uint64_t)lo << 32) | hi);
  }
  std::sort(jointed_pairs.begin(), jointed_pairs.end());
  std::vector<std::vector<Contact>> per_pair(pairs.size());
  auto narrow = [&](size_t p) {
    uint32_t i = pairs[p].first, j = pairs[p].second;
    const Collider& ca = colliders[i];
    const Collider& cb = colliders[j];
    if (ca.body == cb.body) return;
    {
      uint32_t lo = std::min(ca.body, cb.body), hi = std::max(ca.body, cb.body);
      if (std::binary_search(jointed_pairs.begin(), jointed_pairs.end(), ((uint64_t)lo << 32) | hi)) return;
    }
    float reach = sweep[i] + sweep[j] - kMargin;
    Manifold m;
    if (collide_shapes(ca.shape, Iso{pos[ca.body], rot[ca.body]}, cb.shape, Iso{pos[cb.body], rot[cb.body]}, reach, &m)) {
      for (int k = 0; k < m.len; ++k)
        per_pair[p].push_back(Contact{i, j, m.pts[k].position, m.pts[k].normal, m.pts[k].penetration - reach + kMargin, -1, 0.0f});
    }
  };
#ifdef _OPENMP
  if (threads > 1 && pairs.size() >= 64) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (long p = 0; p < (long)pairs.size(); ++p) narrow((size_t)p);
  } else
#endif
    for (size_t p = 0; p < pairs.size(); ++p) narrow(p);
  std::vector<Contact> raw;
  for (auto& v : per_pair) raw.insert(raw.end(), v.begin(), v.end());
  if (has_hf) {
    std::vector<std::vector<Contact>> per_col(ncol);
    auto env_one = [&](uint32_t ci) {
      const Collider& c = colliders[ci];
      std::vector<Shape> tris;
      hf_query(hf, c.aabb, tris);
      for (auto& t : tris) {
        Manifold m;
        if (collide_shapes(c.shape, Iso{pos[c.body], rot[c.body]}, t, Iso{V3{0, 0, 0}, kQId}, sweep[ci], &m)) {
          for (int k = 0; k < m.len; ++k)
            per_col[ci].push_back(Contact{ci, kTerrain, m.pts[k].position, m.pts[k].normal, m.pts[k].penetration - sweep[ci] + kMargin, (int32_t)hf.mat, 0.0f});
        }
      }
    };
#ifdef _OPENMP
    if (threads > 1 && ncol >= 64) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
      for (long c = 0; c < (long)ncol; ++c) env_one((uint32_t)c);
    } else
#endif
      for (uint32_t c = 0; c < ncol; ++c) env_one(c);
    for (auto& v : per_col) raw.insert(raw.end(), v.begin(), v.end());
  }
  // --- Stage 3: cull_and_orient_contacts (step.rs:499-542)
  std::vector<Contact> contacts;
  {
    std::vector<uint32_t> idx(raw.size());
    std::iota(idx.begin(), idx.end(), 0u);
    auto key = [&](uint32_t k) {
      uint32_t a = raw[k].a_collider, b = raw[k].b_collider;
      return a <= b ? std::make_pair(a, b) : std::make_pair(b, a);
    };
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return key(x) < key(y); });
    size_t s = 0;
    while (s < idx.size()) {
      size_t e = s;
      while (e < idx.size() && key(idx[e]) == key(idx[s])) ++e;
      std::vector<Contact> v;
      for (size_t k = s; k < e; ++k) v.push_back(raw[idx[k]]);
      if (v.size() <= 4) contacts.insert(contacts.end(), v.begin(), v.end());
      else if (colliders[v[0].a_collider].shape.kind == SH_BOX) {
        std::vector<float> dep(v.size()); std::vector<V3> pt(v.size());
        size_t deep = 0;
        for (size_t i = 0; i < v.size(); ++i) { dep[i] = v[i].depth; pt[i] = v[i].point; }
        for (size_t i = 1; i < v.size(); ++i) if (sort_key6(v[i].depth) > sort_key6(v[deep].depth)) deep = i;
        int out[4];
        int r = reduce_to_4(dep.data(), pt.data(), (int)v.size(), v[deep].normal, out);
        for (int k = 0; k < r; ++k) contacts.push_back(v[out[k]]);
      } else {
        std::stable_sort(v.begin(), v.end(), [](const Contact& x, const Contact& y) { return sort_key6(x.depth) > sort_key6(y.depth); });
        v.resize(4);
        contacts.insert(contacts.end(), v.begin(), v.end());
      }
      s = e;
    }
    for (auto& c : contacts) {
      if (c.b_collider == kTerrain) continue;
      V3 pa = pos[colliders[c.a_collider].body], pb = pos[colliders[c.b_collider].body];
      if (dot(c.normal, sub(pb, pa)) < 0.0f) c.normal = neg(c.normal);
    }
  }
  const uint32_t nc = (uint32_t)contacts.size();
  stats.contacts = nc;
  // bodies in any joint (solver.rs:483-491, step.rs:160-170)
  std::vector<uint8_t> jointed(count, 0);
  for (auto& jt : joints) { jointed[jt.a] = 1; jointed[jt.b] = 1; }
  // --- islands (islands.rs:27-93): the count, whether the solve runs, the joints' order
  uint32_t n_islands = 0;
  std::vector<uint32_t> active_joints;
  {
    std::vector<uint32_t> parent(count), rank(count, 0), lookup(count, 0xFFFFFFFFu);
    std::iota(parent.begin(), parent.end(), 0u);
    auto find = [&](uint32_t i) {
      uint32_t r = i;
      while (parent[r] != r) { parent[r] = parent[parent[r]]; r = parent[r]; }
      return r;
    };
    auto isdyn = [&](uint32_t id) { return inv_mass[id] > 0.0f; };
    auto unite = [&](uint32_t a, uint32_t b) {
      uint32_t ri = find(a), rj = find(b);
      if (ri != rj) {
        if (rank[ri] < rank[rj]) parent[ri] = rj;
        else if (rank[ri] > rank[rj]) parent[rj] = ri;
        else { parent[ri] = rj; rank[rj] += 1; }
      }
    };
    for (auto& jt : joints)
      if (isdyn(jt.a) && isdyn(jt.b)) unite(jt.a, jt.b);
    for (auto& c : contacts) {
      if (c.b_collider == kTerrain) continue;
      uint32_t a = colliders[c.a_collider].body, b = colliders[c.b_collider].body;
      if (isdyn(a) && isdyn(b)) unite(a, b);
    }
    // active joints (solver.rs:646-648): islands in root order, each island's joints in index order
    std::vector<std::pair<uint32_t, uint32_t>> jorder;
    for (uint32_t k = 0; k < (uint32_t)joints.size(); ++k) {
      const Joint& jt = joints[k];
      bool da = isdyn(jt.a), db = isdyn(jt.b);
      if (!da && !db) continue;
      uint32_t root = da ? find(jt.a) : find(jt.b);
      if (lookup[root] == 0xFFFFFFFFu) lookup[root] = n_islands++;
      jorder.push_back({root, k});
    }
    std::stable_sort(jorder.begin(), jorder.end(), [](auto& x, auto& y) { return x.first < y.first; });
    for (auto& x : jorder) active_joints.push_back(x.second);
    for (auto& c : contacts) {
      uint32_t a = colliders[c.a_collider].body;
      uint32_t b = 0; bool db = false;
      if (c.b_collider != kTerrain) { b = colliders[c.b_collider].body; db = isdyn(b); }
      bool da = isdyn(a);
      if (!da && !db) continue;
      uint32_t root = da ? find(a) : find(b);
      if (lookup[root] == 0xFFFFFFFFu) lookup[root] = n_islands++;
    }
  }
  stats.islands = n_islands;
  std::vector<uint8_t> contact_loaded(count, 0);
  std::vector<std::pair<V3, V3>> bounce_pseudo;  // W6 pseudo-velocities (empty: none this tick)
  std::vector<uint32_t> levels_out(nc, 0xFFFFFFFFu);
  const V3 up = len2(gravity) > 0.0f ? neg(normalize(gravity)) : V3{0, 1, 0};
  std::vector<CC> cons;
  std::vector<std::vector<uint32_t>> batches;
  std::vector<uint32_t> level;
  // the contacts in the order the order-dependent contact passes visit them (warm-start
  // application, ballistic test, position projection): contact order, or in coloured mode the
  // scheduled contacts colour by colour, then the rest
  std::vector<uint32_t> pass_order, pass_rank;
  if (n_islands > 0) {
    // --- solve_islands_parallel (solver.rs:477-1271)
    const float beta = 0.05f, slop = 0.005f, margin = kMargin;
    cons.resize(nc);
    for (uint32_t k = 0; k < nc; ++k) {  // 1. constraint pre-processing (:494-590)
      const Contact& c = contacts[k];
      CC& cs = cons[k];
      cs.ai = colliders[c.a_collider].body;
      cs.terrain = c.b_collider == kTerrain;
      cs.bi = cs.terrain ? 0 : colliders[c.b_collider].body;
      bool a_aw = awake[cs.ai] != 0, b_aw = cs.terrain ? false : awake[cs.bi] != 0;
      cs.inv_a = a_aw ? inv_mass[cs.ai] : 0.0f;
      cs.inv_b = b_aw ? inv_mass[cs.bi] : 0.0f;
      cs.ii_a = cs.inv_a > 0.0f ? inv_inertia_world(cs.ai) : mzero();
      cs.ii_b = cs.inv_b > 0.0f ? inv_inertia_world(cs.bi) : mzero();
      uint32_t mb = cs.terrain ? (uint32_t)(c.env_mat < 0 ? 0 : c.env_mat) : colliders[c.b_collider].mat;
      PairProps pp = pair_props(colliders[c.a_collider].mat, mb);
      cs.n = c.normal;
      orthonormal_basis(cs.n, &cs.t1, &cs.t2);
      cs.ra = sub(c.point, pos[cs.ai]);
      cs.rb = cs.terrain ? V3{0, 0, 0} : sub(c.point, pos[cs.bi]);
      cs.m_n = eff_mass(cs.inv_a, cs.inv_b, cs.ii_a, cs.ii_b, cs.ra, cs.rb, cs.n);
      cs.m_t1 = eff_mass(cs.inv_a, cs.inv_b, cs.ii_a, cs.ii_b, cs.ra, cs.rb, cs.t1);
      cs.m_t2 = eff_mass(cs.inv_a, cs.inv_b, cs.ii_a, cs.ii_b, cs.ra, cs.rb, cs.t2);
      cs.mu_s = pp.mu_s; cs.mu_k = pp.mu_k; cs.sv = rmax(pp.stribeck_v, 1.0e-4f);
      cs.soft = pp.stiffness > 0.0f;
      cs.restitution_bias = 0.0f;
      cs.toi = false;
      float pen = c.depth - margin;
      cs.depth_bias = pen > 0.0f ? rmin(rmax(pen - slop, 0.0f) * (beta / dt), 2.0f) : pen / dt;
      V3 va_l = pre_lin[cs.ai], va_a = pre_ang[cs.ai];
      V3 vb_l = cs.terrain ? V3{0, 0, 0} : pre_lin[cs.bi], vb_a = cs.terrain ? V3{0, 0, 0} : pre_ang[cs.bi];
      float v_pre = dot(sub(add(vb_l, cross(vb_a, cs.rb)), add(va_l, cross(va_a, cs.ra))), cs.n);
      float v_rel_n = 0.5f * (v_pre + dot(contact_rel_vel(*this, cs), cs.n));
      cs.toi_s0 = cs.toi_e = cs.toi_va0 = cs.toi_va1 = cs.toi_vb0 = cs.toi_vb1 = 0.0f;
      if (v_rel_n < -1.0f) {
        cs.restitution_bias = (-pp.restitution) * v_rel_n;
        cs.toi = !jointed[cs.ai] && (cs.terrain || !jointed[cs.bi]);  // W6: free bodies only
        if (cs.toi) {
          // the integrator's motion model: linear velocity from the end of last step (solver.rs:575-587)
          auto at = [&](V3 l, V3 a, V3 r) { return dot(add(l, cross(a, r)), cs.n); };
          V3 sl_a = cs.ai < last_lin_vel.size() ? last_lin_vel[cs.ai] : pre_lin[cs.ai];
          cs.toi_va0 = at(sl_a, pre_ang[cs.ai], cs.ra);
          cs.toi_va1 = at(lin[cs.ai], ang[cs.ai], cs.ra);
          if (!cs.terrain) {
            V3 sl_b = cs.bi < last_lin_vel.size() ? last_lin_vel[cs.bi] : pre_lin[cs.bi];
            cs.toi_vb0 = at(sl_b, pre_ang[cs.bi], cs.rb);
            cs.toi_vb1 = at(lin[cs.bi], ang[cs.bi], cs.rb);
          }
          cs.toi_s0 = -pen;
          cs.toi_e = pp.restitution;
        }
      }
    }
    // 2a. level schedule (:621-642)
    // 2b. joint rows (:644-664), in active order, one contiguous range per joint
    std::vector<JRow> jrows;
    std::vector<std::pair<uint32_t, uint32_t>> jrange(joints.size(), {0u, 0u});
    for (uint32_t jk : active_joints) {
      uint32_t s = (uint32_t)jrows.size();
      joint_rows(*this, joints[jk], jk, dt, jrows);
      jrange[jk] = {s, (uint32_t)jrows.size()};
      for (uint32_t k = s; k < (uint32_t)jrows.size(); ++k) jrows[k].idx = (uint8_t)(k - s);
      if (jrows.size() > s) jrows[s].cnt = (uint8_t)(jrows.size() - s);
    }
    const uint32_t njr = (uint32_t)jrows.size();
    std::vector<float> jacc(njr, 0.0f);
    // 2a. one level schedule (:621-642, 666-683) over the joint rows, then the contact rows: entry
    // e < njr is joint row e, entry njr + k contact k. Every sweep then runs an island's joint rows
    // before its contacts, as the reference's joint batches run before its contact batches. A
    // joint's rows form one unit (its level, run in order by its first row), as a joint is one task
    // of the reference's joint batches. A contact's side on a sleeping jointed body is read-only for
    // the contact but moved by that body's joint rows, so the schedule and the solve islands count
    // it as touched.
    auto ent = [&](uint32_t e, uint32_t* a, uint32_t* b, bool* ta, bool* tb) {
      if (e < njr) {
        const JRow& r = jrows[e];
        *a = r.a; *b = r.b; *ta = r.wa > 0.0f; *tb = r.wb > 0.0f;
        return true;
      }
      const CC& c = cons[e - njr];
      *a = c.ai; *b = c.bi;
      *ta = c.inv_a > 0.0f || (jointed[c.ai] && inv_mass[c.ai] > 0.0f);
      *tb = !c.terrain && (c.inv_b > 0.0f || (jointed[c.bi] && inv_mass[c.bi] > 0.0f));
      return c.inv_a > 0.0f || (!c.terrain && c.inv_b > 0.0f);
    };
    const uint32_t nent = njr + nc;
    std::vector<uint32_t> ent_level(nent, 0xFFFFFFFFu);
    {
      std::vector<uint32_t> bl(count, 0);
      batches.clear();
      for (uint32_t e = 0; e < nent; ++e) {
        uint32_t a, b; bool ta, tb;
        if (!ent(e, &a, &b, &ta, &tb)) continue;
        if (e < njr && jrows[e].idx) {  // a joint's later row: with its first
          uint32_t t = ent_level[e - jrows[e].idx];
          batches[t].push_back(e);
          ent_level[e] = t;
          continue;
        }
        uint32_t la = ta ? bl[a] : 0, lb = tb ? bl[b] : 0;
        uint32_t t = la > lb ? la : lb;
        if (t >= batches.size()) batches.emplace_back();
        batches[t].push_back(e);
        ent_level[e] = t;
        if (ta) bl[a] = t + 1;
        if (tb) bl[b] = t + 1;
      }
    }
    // Coloured order (an extension; worlds without joints). Each solve island -- rows joined
    // through the bodies they write -- is coloured by first fit in level order: walking the levels,
    // a row takes the smallest colour that no already coloured row writing one of its bodies holds
    // (128 colours per body at most). Rows of one colour then share no written body. An island
    // with a row that finds no free colour keeps its levels, and so does an island of more than
    // 32 rows whose colours are no fewer than its levels. Every pass that follows the level
    // schedule in the serial order then visits the rows colour by colour (within a colour in
    // (level, serial) order, which changes nothing: the rows of a colour are independent), so the
    // Gauss-Seidel updates are reordered and the results are no longer the reference's bits.
    if (coloured && njr == 0 && !batches.empty()) {
      std::vector<uint32_t> root(count);
      std::iota(root.begin(), root.end(), 0u);
      auto find = [&](uint32_t x) {
        while (root[x] != x) { root[x] = root[root[x]]; x = root[x]; }
        return x;
      };
      for (auto& b : batches)
        for (uint32_t e : b) {
          uint32_t a, bb; bool ta, tb;
          ent(e, &a, &bb, &ta, &tb);
          if (ta && tb) {
            uint32_t ra = find(a), rb = find(bb);
            if (ra != rb) root[ra < rb ? rb : ra] = ra < rb ? ra : rb;
          }
        }
      std::vector<uint64_t> mask(2 * (size_t)count, 0ull);
      std::vector<uint32_t> colour(nent, 0xFFFFFFFFu);
      std::vector<uint8_t> over(count, 0);
      for (auto& b : batches)
        for (uint32_t e : b) {
          uint32_t a, bb; bool ta, tb;
          ent(e, &a, &bb, &ta, &tb);
          uint64_t m0 = 0, m1 = 0;
          if (ta) { m0 |= mask[2 * a]; m1 |= mask[2 * a + 1]; }
          if (tb) { m0 |= mask[2 * bb]; m1 |= mask[2 * bb + 1]; }
          uint32_t c = 0xFFFFFFFFu;
          if (~m0) c = (uint32_t)__builtin_ctzll(~m0);
          else if (~m1) c = 64u + (uint32_t)__builtin_ctzll(~m1);
          colour[e] = c;
          if (c == 0xFFFFFFFFu) { over[find(ta ? a : bb)] = 1; continue; }
          const uint64_t bit = 1ull << (c & 63u);
          if (ta) mask[2 * a + (c >> 6)] |= bit;
          if (tb) mask[2 * bb + (c >> 6)] |= bit;
        }
      // an island of more than 32 rows (the size the device solves as a group alone) that needs no
      // fewer colours than levels keeps its levels too
      std::vector<uint32_t> nrow(count, 0), ncol(count, 0), nlev(count, 0);
      for (uint32_t L = 0; L < (uint32_t)batches.size(); ++L)
        for (uint32_t e : batches[L]) {
          uint32_t a, bb; bool ta, tb;
          ent(e, &a, &bb, &ta, &tb);
          uint32_t r = find(ta ? a : bb);
          nrow[r]++;
          nlev[r] = std::max(nlev[r], L + 1);
          if (colour[e] != 0xFFFFFFFFu) ncol[r] = std::max(ncol[r], colour[e] + 1);
        }
      for (uint32_t r = 0; r < count; ++r)
        if (nrow[r] > 32u && ncol[r] >= nlev[r]) over[r] = 1;
      std::vector<std::vector<uint32_t>> cb;
      for (uint32_t L = 0; L < (uint32_t)batches.size(); ++L)
        for (uint32_t e : batches[L]) {
          uint32_t a, bb; bool ta, tb;
          ent(e, &a, &bb, &ta, &tb);
          uint32_t key = over[find(ta ? a : bb)] ? L : colour[e];
          if (key >= cb.size()) cb.resize(key + 1);
          cb[key].push_back(e);
          ent_level[e] = key;
        }
      batches.swap(cb);
    }
    stats.levels = (uint32_t)batches.size();
    for (auto& b : batches) stats.max_batch = std::max<uint32_t>(stats.max_batch, (uint32_t)b.size());
    for (uint32_t k = 0; k < nc; ++k) levels_out[k] = ent_level[njr + k];
    pass_order.clear();
    pass_rank.assign(nc, 0xFFFFFFFFu);
    if (coloured && njr == 0) {
      for (auto& b : batches)
        for (uint32_t e : b) { pass_rank[e] = (uint32_t)pass_order.size(); pass_order.push_back(e); }
      for (uint32_t k = 0; k < nc; ++k)
        if (pass_rank[k] == 0xFFFFFFFFu) { pass_rank[k] = (uint32_t)pass_order.size(); pass_order.push_back(k); }
    } else {
      for (uint32_t k = 0; k < nc; ++k) { pass_rank[k] = k; pass_order.push_back(k); }
    }
    // warm start, joints (:699-712): serial in joint order, clamped to each row's bounds; distance
    // rows start cold (:704-705)
    for (uint32_t jk = 0; jk < (uint32_t)joints.size(); ++jk) {
      uint32_t s = jrange[jk].first, e = jrange[jk].second;
      if (e == s || joints[jk].kind != 0 || jrows[s].carrier) continue;
      auto it = warm_joints.find(jk);
      if (it == warm_joints.end()) continue;
      const WarmJointRows& prev = it->second;
      if (prev.size() != e - s) continue;
      bool same = true;
      for (uint32_t k = s; k < e; ++k) same = same && prev[k - s].first == jrows[k].tag;
      if (!same) continue;
      for (uint32_t k = s; k < e; ++k) {
        float lam = clampf(prev[k - s].second, jrows[k].lam_min, jrows[k].lam_max);
        jacc[k] = lam;
        if (lam != 0.0f) joint_row_apply(*this, jrows[k], lam);
      }
    }
    std::vector<float> acc_jn(nc, 0.0f), acc_jt(2 * (size_t)nc, 0.0f);
    // 3. warm start (:717-762)
    std::vector<WarmKey> keys(nc);
    std::vector<V3> anchors(nc);
    for (uint32_t k = 0; k < nc; ++k) {
      const Contact& c = contacts[k];
      uint32_t ba = colliders[c.a_collider].body;
      keys[k] = c.b_collider == kTerrain ? WarmKey{ba, 0xFFFFFFFFu, 0u, 0u} : WarmKey{ba, colliders[c.b_collider].body, 0u, 0u};
      anchors[k] = qrot(qconj(rot[cons[k].ai]), sub(c.point, pos[cons[k].ai]));
    }
    {
      std::map<WarmKey, std::vector<bool>> used;
      const float tol2 = kWarmTol * kWarmTol;
      std::vector<float> ref_jn(nc, 0.0f);
      std::vector<V3> ref_jt(nc, V3{0, 0, 0});
      std::vector<uint8_t> ref_have(nc, 0);
      for (uint32_t k = 0; k < nc; ++k) {
        const CC& cs = cons[k];
        if (cs.soft) continue;
        auto it = warm.find(keys[k]);
        if (it == warm.end()) continue;
        const auto& entries = it->second;
        auto& taken = used.emplace(keys[k], std::vector<bool>(entries.size(), false)).first->second;
        bool have = false; float bd = 0; size_t bk = 0;
        for (size_t e = 0; e < entries.size(); ++e) {
          if (taken[e]) continue;
          float d = len2(sub(entries[e].la, anchors[k]));
          if (d <= tol2 && (!have || d < bd)) { have = true; bd = d; bk = e; }
        }
        if (!have) continue;
        taken[bk] = true;
        stats.warm_matched++;
        ref_jn[k] = entries[bk].jn;
        ref_jt[k] = entries[bk].jt;
        ref_have[k] = 1;
      }
      // application in contact order (solver.rs:749-760); with predictions offered (the learned
      // warm start), each row keeps the start -- the previous tick's impulse or none, against the
      // prediction -- that leaves the smaller normal velocity error |bias - v_rel . n|
      const bool preds = next_pred.size() >= 4 * (size_t)nc;
      auto apply_start = [&](const CC& cs, float jn, V3 jt, float* out_jn, float* out_t) {
        V3 imp = mul(cs.n, jn);
        float mu = mu_dynamic(cs, slip_speed(*this, cs));
        V3 t = clamp_length_max(V3{dot(jt, cs.t1), dot(jt, cs.t2), 0.0f}, mu * jn);
        if (out_jn) { *out_jn = jn; out_t[0] = t.x; out_t[1] = t.y; }
        imp = add(imp, add(mul(cs.t1, t.x), mul(cs.t2, t.y)));
        apply_contact_impulse(*this, cs, imp);
      };
      auto trial_err = [&](const CC& cs, bool apply, float jn, V3 jt) {
        V3 la = lin[cs.ai], aa = ang[cs.ai], lb{}, ab{};
        if (!cs.terrain) { lb = lin[cs.bi]; ab = ang[cs.bi]; }
        if (apply) apply_start(cs, jn, jt, nullptr, nullptr);
        float e = std::fabs(cs.depth_bias - dot(contact_rel_vel(*this, cs), cs.n));
        lin[cs.ai] = la; ang[cs.ai] = aa;
        if (!cs.terrain) { lin[cs.bi] = lb; ang[cs.bi] = ab; }
        return e;
      };
      for (uint32_t k : pass_order) {
        const CC& cs = cons[k];
        if (cs.soft) continue;
        const bool hp = preds && next_pred[4 * (size_t)k + 3] != 0.0f;
        if (!ref_have[k] && !hp) continue;
        if (hp) {
          const float su = cs.m_n * kImpulseUnit;
          float pjn = rmax(next_pred[4 * (size_t)k] * su, 0.0f);
          V3 pjt = add(mul(cs.t1, next_pred[4 * (size_t)k + 1] * su), mul(cs.t2, next_pred[4 * (size_t)k + 2] * su));
          float e_ref = trial_err(cs, ref_have[k] != 0, ref_jn[k], ref_jt[k]);
          float e_pred = trial_err(cs, true, pjn, pjt);
          if (e_pred < e_ref) {
            apply_start(cs, pjn, pjt, &acc_jn[k], &acc_jt[2 * k]);
            stats.pred_used++;
            continue;
          }
        }
        if (ref_have[k]) apply_start(cs, ref_jn[k], ref_jt[k], &acc_jn[k], &acc_jt[2 * k]);
      }
      next_pred.clear();
    }
    // iterations (:788-915)
    // Residual stop (an extension; the reference always runs iters_v sweeps): each solve island --
    // the rows joined through the bodies they move -- sweeps until the largest velocity change one
    // of its rows made in a sweep is <= res_tol, or the cap. Islands share no body, so stopping one
    // early leaves every other island's arithmetic unchanged.
    std::vector<uint32_t> sroot(count);
    std::iota(sroot.begin(), sroot.end(), 0u);
    auto sfind = [&](uint32_t x) {
      while (sroot[x] != x) { sroot[x] = sroot[sroot[x]]; x = sroot[x]; }
      return x;
    };
    for (auto& b : batches)
      for (uint32_t e : b) {
        uint32_t a, bb; bool ta, tb;
        ent(e, &a, &bb, &ta, &tb);
        if (ta && tb) {
          uint32_t ra = sfind(a), rb = sfind(bb);
          if (ra != rb) sroot[ra < rb ? rb : ra] = ra < rb ? ra : rb;
        }
      }
    std::vector<uint32_t> row_isl(nent, 0xFFFFFFFFu), isl_of_root(count, 0xFFFFFFFFu);
    uint32_t n_sisl = 0;
    for (auto& b : batches)
      for (uint32_t e : b) {
        uint32_t a, bb; bool ta, tb;
        ent(e, &a, &bb, &ta, &tb);
        uint32_t r = sfind(ta ? a : bb);
        if (isl_of_root[r] == 0xFFFFFFFFu) isl_of_root[r] = n_sisl++;
        row_isl[e] = isl_of_root[r];
      }
    std::vector<float> row_res(nent, 0.0f), isl_last(n_sisl, 0.0f);
    std::vector<uint32_t> isl_sweeps(n_sisl, 0), isl_rows(n_sisl, 0);
    std::vector<uint8_t> isl_done(n_sisl, 0);
    for (auto& b : batches)
      for (uint32_t e : b) isl_rows[row_isl[e]]++;
    auto row = [&](uint32_t k, float* resid) {
      const CC& cs = cons[k];
      float v_rel_n = dot(contact_rel_vel(*this, cs), cs.n);
      float jn_raw = (cs.depth_bias - v_rel_n) * cs.m_n;
      float old_jn = acc_jn[k];
      float new_jn = rmax(old_jn + jn_raw, 0.0f);
      acc_jn[k] = new_jn;
      apply_contact_impulse(*this, cs, mul(cs.n, new_jn - old_jn));
      V3 vf = contact_rel_vel(*this, cs);
      float vt1 = dot(vf, cs.t1), vt2 = dot(vf, cs.t2);
      float slip = std::sqrt(vt1 * vt1 + vt2 * vt2);
      float mu = mu_dynamic(cs, slip);
      V3 old_t{acc_jt[2 * k], acc_jt[2 * k + 1], 0.0f};
      V3 new_t = clamp_length_max(sub(old_t, V3{vt1 * cs.m_t1, vt2 * cs.m_t2, 0.0f}), mu * new_jn);
      acc_jt[2 * k] = new_t.x; acc_jt[2 * k + 1] = new_t.y;
      V3 d = sub(new_t, old_t);
      apply_contact_impulse(*this, cs, add(mul(cs.t1, d.x), mul(cs.t2, d.y)));
      // residual: velocity change this row made (m/s)
      float r = 0.0f;
      if (cs.m_n > 0.0f) r = rmax(r, std::fabs(new_jn - old_jn) / cs.m_n);
      if (cs.m_t1 > 0.0f) r = rmax(r, std::fabs(d.x) / cs.m_t1);
      if (cs.m_t2 > 0.0f) r = rmax(r, std::fabs(d.y) / cs.m_t2);
      *resid = rmax(*resid, r);
    };
    // one entry: a joint row (solver.rs:821-830; residual |delta lambda| / m_eff) or a contact
    auto solve_ent = [&](uint32_t e, float* resid) {
      if (e < njr) {  // the first row of a joint runs the joint's rows in order
        for (uint32_t q = 0; q < jrows[e].cnt; ++q) {
          float d = joint_row_update(*this, jrows[e + q], jacc[e + q]);
          float r = std::fabs(d) / jrows[e + q].m_eff;
          if (q == 0) *resid = rmax(*resid, r);
          else row_res[e + q] = r;
        }
      } else {
        row(e - njr, resid);
      }
    };
    const bool residual_mode = res_tol > 0.0f;
    const uint32_t max_sweeps = residual_mode ? (res_max > 0 ? res_max : iters_v) : iters_v;
    // Each solve island sweeps on its own: its rows in batch order (the serial order restricted to
    // the island), until its residual stop or the cap. Islands move disjoint bodies, so solving
    // them one after another, or on several threads at once, gives the bits of the batch-by-batch
    // sweep over all islands.
    std::vector<uint32_t> isl_first(n_sisl + 1, 0), isl_list(nent);
    for (uint32_t i = 0; i < n_sisl; ++i) isl_first[i + 1] = isl_first[i] + isl_rows[i];
    {
      std::vector<uint32_t> fill(isl_first.begin(), isl_first.end() - 1);
      for (auto& b : batches)
        for (uint32_t e : b) isl_list[fill[row_isl[e]]++] = e;
    }
    std::vector<std::vector<float>> isl_hist(diag_worst ? n_sisl : 0);
    auto solve_island = [&](uint32_t i) {
      const uint32_t* L = isl_list.data() + isl_first[i];
      const uint32_t n = isl_first[i + 1] - isl_first[i];
      for (uint32_t it = 0; it < max_sweeps; ++it) {
        for (uint32_t q = 0; q < n; ++q) {
          uint32_t e = L[q];
          if (e < njr && jrows[e].idx) continue;
          row_res[e] = 0.0f;
          solve_ent(e, &row_res[e]);
        }
        float r = 0.0f;
        for (uint32_t q = 0; q < n; ++q) r = rmax(r, row_res[L[q]]);
        isl_sweeps[i] = it + 1;
        isl_last[i] = r;
        if (diag_worst) isl_hist[i].push_back(r);
        if (residual_mode && r <= res_tol) { isl_done[i] = 1; break; }
      }
    };
#ifdef _OPENMP
    if (threads > 1) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
      for (long i = 0; i < (long)n_sisl; ++i) solve_island((uint32_t)i);
    } else
#endif
      for (uint32_t i = 0; i < n_sisl; ++i) solve_island(i);
    if (diag_worst) {
      diag_rows.clear();
      diag_hist.clear();
      uint32_t worst = 0;
      for (uint32_t i = 1; i < n_sisl; ++i)
        if (isl_last[i] > isl_last[worst]) worst = i;
      if (n_sisl) {
        diag_hist = isl_hist[worst];
        for (uint32_t q = isl_first[worst]; q < isl_first[worst + 1]; ++q) {
          uint32_t e = isl_list[q];
          uint32_t a = 0xFFFFFFFFu, bb = 0xFFFFFFFFu;
          float mn = 0.0f, jn = 0.0f;
          if (e >= njr) { const CC& cs = cons[e - njr]; a = cs.ai; bb = cs.terrain ? 0xFFFFFFFFu : cs.bi; mn = cs.m_n; jn = acc_jn[e - njr]; }
          float fa, fb;
          std::memcpy(&fa, &a, 4); std::memcpy(&fb, &bb, 4);
          diag_rows.insert(diag_rows.end(), {fa, fb, mn, jn, row_res[e]});
        }
      }
    }
    stats.sweeps = 0;
    stats.residual = 0.0f;
    stats.rows_scheduled = 0;
    stats.row_sweeps = 0;
    for (uint32_t i = 0; i < n_sisl; ++i) {
      stats.sweeps = std::max(stats.sweeps, isl_sweeps[i]);
      stats.residual = rmax(stats.residual, isl_last[i]);
      stats.rows_scheduled += isl_rows[i];
      stats.row_sweeps += isl_rows[i] * isl_sweeps[i];
      if (residual_mode && !isl_done[i]) { stats.islands_capped++; stats.rows_capped += isl_rows[i]; }
      stats.res_hist[res_bin(isl_last[i])]++;
    }
    // joints solved this tick replace their rows; the rest keep theirs (:946-952); distance rows
    // are not kept
    for (uint32_t jk = 0; jk < (uint32_t)joints.size(); ++jk) {
      uint32_t s = jrange[jk].first, e = jrange[jk].second;
      if (e == s || joints[jk].kind != 0 || jrows[s].carrier) continue;
      WarmJointRows rows;
      for (uint32_t k = s; k < e; ++k) rows.push_back({jrows[k].tag, jacc[k]});
      warm_joints[jk] = rows;
    }
    // warm-start cache (:917-944)
    std::map<WarmKey, std::vector<WarmContact>> nw;
    for (uint32_t k = 0; k < nc; ++k) {
      const CC& cs = cons[k];
      if (cs.soft) continue;
      V3 jt = add(mul(cs.t1, acc_jt[2 * k]), mul(cs.t2, acc_jt[2 * k + 1]));
      if (acc_jn[k] == 0.0f && vzero(jt)) continue;
      nw[keys[k]].push_back(WarmContact{anchors[k], acc_jn[k], jt});
    }
    auto idle = [&](uint32_t b) {
      return b == 0xFFFFFFFFu || ((b < alive.size() && alive[b] != 0) && (!dyn[b] || !awake[b]));
    };
    for (auto& kv : warm)
      if (idle(std::get<0>(kv.first)) && idle(std::get<1>(kv.first)) && nw.find(kv.first) == nw.end()) nw[kv.first] = kv.second;
    warm.swap(nw);
    // 3a. shock propagation (:964-993)
    {
      auto height = [&](const CC& cs) {
        float ha = dot(pos[cs.ai], up);
        return cs.terrain ? -INFINITY : rmin(ha, dot(pos[cs.bi], up));
      };
      std::vector<uint32_t> ord;
      for (uint32_t k = 0; k < nc; ++k)
        if (!cons[k].soft && (cons[k].inv_a > 0.0f || cons[k].inv_b > 0.0f)) ord.push_back(k);
      std::vector<int64_t> hk(nc);
      for (uint32_t k : ord) hk[k] = sort_key6(height(cons[k]));
      std::sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) { return hk[x] != hk[y] ? hk[x] < hk[y] : x < y; });
      for (uint32_t k : ord) {
        CC cs = cons[k];
        if (cs.inv_a > 0.0f && cs.inv_b > 0.0f) {
          if (dot(pos[cs.ai], up) < dot(pos[cs.bi], up)) { cs.inv_a = 0.0f; cs.ii_a = mzero(); }
          else { cs.inv_b = 0.0f; cs.ii_b = mzero(); }
          cs.m_n = eff_mass(cs.inv_a, cs.inv_b, cs.ii_a, cs.ii_b, cs.ra, cs.rb, cs.n);
        }
        float v = dot(contact_rel_vel(*this, cs), cs.n);
        float old = acc_jn[k];
        float nw2 = rmax(old + (cs.depth_bias - v) * cs.m_n, 0.0f);
        acc_jn[k] = nw2;
        apply_contact_impulse(*this, cs, mul(cs.n, nw2 - old));
      }
    }
    // 3b. restitution (:1001-1008): toi rows skip it; without joints every bouncing row is toi
    for (uint32_t k = 0; k < nc; ++k) {
      const CC& cs = cons[k];
      if (cs.toi || cs.restitution_bias <= 0.0f || acc_jn[k] <= 0.0f) continue;
      float v = dot(contact_rel_vel(*this, cs), cs.n);
      float old = acc_jn[k];
      float nw2 = rmax(old + (cs.restitution_bias - v) * cs.m_n, 0.0f);
      acc_jn[k] = nw2;
      apply_contact_impulse(*this, cs, mul(cs.n, nw2 - old));
    }
    // W6 bounce passes (:1009-1241)
    w6_bounce(*this, cons, acc_jn, acc_jt, jointed, dt, count, bounce_pseudo, &stats.bounce_rows);
    // contact_loaded (:1248-1256) and impulse write-back (:1268-1270)
    for (uint32_t k = 0; k < nc; ++k) {
      const CC& cs = cons[k];
      bool loaded = acc_jn[k] > 0.0f || acc_jt[2 * k] != 0.0f || acc_jt[2 * k + 1] != 0.0f;
      if (loaded) { contact_loaded[cs.ai] = 1; if (!cs.terrain) contact_loaded[cs.bi] = 1; }
      contacts[k].impulse = acc_jn[k];
    }
  }
  // --- Stage 4: integration (step.rs:154-280)
  std::vector<Iso> original(count, Iso{V3{0, 0, 0}, kQId}), predicted(count, Iso{V3{0, 0, 0}, kQId});
  std::vector<uint8_t> constrained(count, 0);
  for (auto& c : contacts) {
    constrained[colliders[c.a_collider].body] = 1;
    if (c.b_collider != kTerrain) constrained[colliders[c.b_collider].body] = 1;
  }
  for (auto& jt : joints) { constrained[jt.a] = 1; constrained[jt.b] = 1; }
  std::vector<uint8_t> ballistic(count);
  for (uint32_t i = 0; i < count; ++i) ballistic[i] = !constrained[i] || (!jointed[i] && !contact_loaded[i]);
  for (uint32_t ci = 0; ci < nc; ++ci) {
    const Contact& c = contacts[pass_order.size() == nc ? pass_order[ci] : ci];
    uint32_t a = colliders[c.a_collider].body;
    bool hb = c.b_collider != kTerrain;
    uint32_t b = hb ? colliders[c.b_collider].body : 0;
    if (!ballistic[a] && (!hb || !ballistic[b])) continue;
    auto moving_lin = [&](uint32_t id) {
      V3 v = lin[id];
      return ballistic[id] ? mul(add(last_lin_vel[id], v), 0.5f) : v;
    };
    V3 la = moving_lin(a), wa = ang[a];
    V3 ra = sub(c.point, pos[a]);
    V3 lb{0, 0, 0}, wb{0, 0, 0}, rb{0, 0, 0};
    if (hb) { lb = moving_lin(b); wb = ang[b]; rb = sub(c.point, pos[b]); }
    float approach = dot(sub(add(lb, cross(wb, rb)), add(la, cross(wa, ra))), c.normal);
    V3 vbl = hb ? lin[b] : V3{0, 0, 0}, vba = hb ? ang[b] : V3{0, 0, 0};
    float v_end = dot(sub(add(vbl, cross(vba, rb)), add(lin[a], cross(ang[a], ra))), c.normal);
    float s0 = -(c.depth - kMargin);
    if (s0 + (2.0f * v_end) * dt < 0.0f || s0 + approach * dt < 0.0f) {
      ballistic[a] = 0;
      if (hb) ballistic[b] = 0;
    }
  }
  for (uint32_t i = 0; i < count; ++i) {
    if (!dyn[i] || !awake[i]) continue;
    Iso pose{pos[i], rot[i]};
    original[i] = pose;
    V3 vl = lin[i], va = ang[i];
    pose.pos = add(pose.pos, mul(vl, dt));
    if (ballistic[i]) pose.pos = add(pose.pos, mul(sub(last_lin_vel[i], vl), 0.5f * dt));
    if (len2(va) > 0.0f) {
      M3 l = inv_inertia_world(i);
      float det = mdet(l);
      bool has_m = fin(det) && std::fabs(det) > 1.0e-20f;
      V3 m = has_m ? mvec(minverse(l), va) : V3{0, 0, 0};
      auto turn = [](Q4 q, V3 w, float h) -> Q4 {
        if (len2(w) <= 1.0e-18f) return q;
        return qnormalize(qmul(qfrom_axis_angle(normalize(w), len(w) * h), q));
      };
      Q4 start = pose.rot;
      pose.rot = turn(start, va, dt);
      if (has_m) {
        M3 il = inv_mass[i] == 0.0f ? mzero() : inv_I[i];
        auto w_at = [&](Q4 q) { M3 r = mfrom_quat(q); return mvec(mmul(mmul(r, il), mtranspose(r)), m); };
        float mean = ((il.c0.x + il.c1.y) + il.c2.z) / 3.0f;
        M3 dev = msub(il, mdiag(splat(mean)));
        bool principal = len(cross(m, va)) < (kTurnPrincipal * len(m)) * len(va);
        float gain = principal ? 0.0f : (dt * rmax(rmax(len(dev.c0), len(dev.c1)), len(dev.c2))) * len(m);
        float cq = std::ceil(gain / kTurnGain);
        long nn = std::isnan(cq) ? 0 : (cq <= 0.0f ? 0 : (cq >= 1.8e19f ? LONG_MAX : (long)cq));
        int n = (int)(nn < 1 ? 1 : (nn > kTurnMaxSplit ? kTurnMaxSplit : nn));
        float h = dt / (float)n;
        Q4 q = start; V3 w = va;
        for (int s = 0; s < n; ++s) {
          Q4 q0 = q;
          q = turn(q0, w, h);
          V3 we = w_at(q);
          for (int r = 0; r < 2; ++r) { q = turn(q0, mul(add(w, we), 0.5f), h); we = w_at(q); }
          w = we;
        }
        pose.rot = q;
        va = w;
        set_vel(i, vl, va);
      }
    }
    // a bounced free body's pseudo-velocity (W6, step.rs:271-277): moves it, never enters its velocity
    if (i < bounce_pseudo.size()) {
      V3 pl = bounce_pseudo[i].first, pa = bounce_pseudo[i].second;
      pose.pos = add(pose.pos, mul(pl, dt));
      if (len2(pa) > 0.0f) pose.rot = qnormalize(qmul(qfrom_axis_angle(normalize(pa), len(pa) * dt), pose.rot));
    }
    set_pose(i, pose);
    predicted[i] = Iso{pos[i], rot[i]};
  }
  // --- Stage 5: position pass (step.rs:284-309, 423-497)
  struct PC { uint32_t a; bool hb; uint32_t b; V3 la, lb, pbw, n; float pen0; uint32_t src; };
  std::vector<PC> pcs;
  {
    auto movable = [&](uint32_t id) { return inv_mass[id] > 0.0f && awake[id] != 0; };
    auto pose_at = [&](uint32_t id) { return (dyn[id] && awake[id]) ? original[id] : Iso{pos[id], rot[id]}; };
    for (uint32_t k = 0; k < nc; ++k) {
      const Contact& c = contacts[k];
      uint32_t a = colliders[c.a_collider].body;
      bool hb = c.b_collider != kTerrain;
      uint32_t b = hb ? colliders[c.b_collider].body : 0;
      if (!movable(a) && !(hb && movable(b))) continue;
      uint32_t mb = hb ? colliders[c.b_collider].mat : (uint32_t)(c.env_mat < 0 ? 0 : c.env_mat);
      if (pair_props(colliders[c.a_collider].mat, mb).stiffness > 0.0f) continue;
      PC pc;
      pc.a = a; pc.hb = hb; pc.b = b; pc.n = c.normal; pc.pen0 = c.depth - kMargin; pc.src = k;
      Iso pa = pose_at(a);
      pc.la = qrot(qconj(pa.rot), sub(c.point, pa.pos));
      if (hb) { Iso pb = pose_at(b); pc.lb = qrot(qconj(pb.rot), sub(c.point, pb.pos)); }
      else pc.lb = V3{0, 0, 0};
      pc.pbw = c.point;
      pcs.push_back(pc);
    }
  }
  std::vector<V3> split_l(count, V3{0, 0, 0}), split_a(count, V3{0, 0, 0});
  auto project = [&](bool shock) {
    std::vector<uint32_t> ord(pcs.size());
    std::iota(ord.begin(), ord.end(), 0u);
    if (!shock && coloured && pass_rank.size() == nc)  // coloured order: the passes' rank of each contact
      std::sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) { return pass_rank[pcs[x].src] < pass_rank[pcs[y].src]; });
    if (shock) {
      std::vector<int64_t> hk(pcs.size());
      for (size_t x = 0; x < pcs.size(); ++x)
        hk[x] = sort_key6(pcs[x].hb ? rmin(dot(pos[pcs[x].a], up), dot(pos[pcs[x].b], up)) : -INFINITY);
      std::sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) { return hk[x] != hk[y] ? hk[x] < hk[y] : x < y; });
    }
    for (uint32_t k : ord) {
      const PC& pc = pcs[k];
      bool am = inv_mass[pc.a] > 0.0f && awake[pc.a];
      bool bm = pc.hb && inv_mass[pc.b] > 0.0f && awake[pc.b];
      if (shock && am && bm) {
        float ha = dot(pos[pc.a], up), hb2 = dot(pos[pc.b], up);
        if (ha < hb2) am = false; else bm = false;
      }
      Iso pa{pos[pc.a], rot[pc.a]};
      V3 wa = add(pa.pos, qrot(pa.rot, pc.la));
      Iso pb{V3{0, 0, 0}, kQId};
      V3 wb;
      if (pc.hb) { pb = Iso{pos[pc.b], rot[pc.b]}; wb = add(pb.pos, qrot(pb.rot, pc.lb)); }
      else wb = pc.pbw;
      float pen = pc.pen0 - dot(sub(wb, wa), pc.n);
      float err = pen - kPosSlop;
      if (err <= 0.0f) continue;
      V3 ra = sub(wa, pa.pos);
      V3 rb = pc.hb ? sub(wb, pb.pos) : V3{0, 0, 0};
      float ima = am ? inv_mass[pc.a] : 0.0f; M3 iia = am ? inv_inertia_world(pc.a) : mzero();
      float imb = (pc.hb && bm) ? inv_mass[pc.b] : 0.0f; M3 iib = (pc.hb && bm) ? inv_inertia_world(pc.b) : mzero();
      V3 ca = cross(ra, pc.n), cb = cross(rb, pc.n);
      float w = ((ima + imb) + dot(ca, mvec(iia, ca))) + dot(cb, mvec(iib, cb));
      if (w <= 1.0e-9f) continue;
      float lambda = err / w;
      auto move_body = [&](uint32_t id, const Iso& pose, float im, const M3& ii, V3 r, V3 j) {
        V3 dth = mvec(ii, cross(r, j));
        split_l[id] = add(split_l[id], mul(j, im));
        split_a[id] = add(split_a[id], dth);
        Q4 dq = qscale(qmul(Q4{dth.x, dth.y, dth.z, 0.0f}, pose.rot), 0.5f);
        Q4 nr = qnormalize(Q4{pose.rot.x + dq.x, pose.rot.y + dq.y, pose.rot.z + dq.z, pose.rot.w + dq.w});
        set_pose(id, Iso{add(pose.pos, mul(j, im)), nr});
      };
      if (am) move_body(pc.a, pa, ima, iia, ra, mul(neg(pc.n), lambda));
      if (pc.hb && bm) move_body(pc.b, pb, imb, iib, rb, mul(pc.n, lambda));
    }
  };
  // joints and contacts interleaved (step.rs:287-308): each sweep the joint pass (SHAKE
  // directions from the step's start poses) then one contact projection
  const bool has_joints = !joints.empty();
  std::vector<Iso> start_poses;
  std::vector<uint8_t> frozen;
  if (has_joints) {
    start_poses.resize(count);
    frozen.resize(count);
    for (uint32_t i = 0; i < count; ++i) {
      start_poses[i] = (dyn[i] && awake[i]) ? original[i] : Iso{pos[i], rot[i]};
      frozen[i] = (!dyn[i] || !awake[i]) ? 1 : 0;
    }
    for (auto& jt : joints) {  // Joints::begin_step (bodies.rs:310-318)
      for (int k = 0; k < 3; ++k) { jt.lam_t[k] = 0.0f; jt.lam_r[k] = 0.0f; }
      jt.lambda_acc = 0.0f;
    }
  }
  if (has_joints || !pcs.empty()) {
    for (uint32_t it = 0; it < iters_p; ++it) {
      if (has_joints) solve_joints_pass(*this, dt, start_poses, frozen);
      project(false);
    }
    project(true);
  }
  // --- Stage 6: velocity from corrections (step.rs:316-379)
  std::vector<uint8_t> touching(count, 0);
  for (auto& c : contacts) {
    if (c.b_collider != kTerrain) continue;
    uint32_t mb = (uint32_t)(c.env_mat < 0 ? 0 : c.env_mat);
    if (c.depth - kMargin > -kPosSlop && pair_props(colliders[c.a_collider].mat, mb).stiffness <= 0.0f)
      touching[colliders[c.a_collider].body] = 1;
  }
  // bodies of a joint with a velocity drive on a rotational axis keep the angular velocity the
  // motor rows gave them (step.rs:352-366, the "motor overwrite")
  std::vector<uint8_t> driven(count, 0);
  for (auto& jt : joints) {
    bool any = false;
    for (int k = 0; k < 3; ++k) any = any || (jt.r[k].has_drive && jt.r[k].vel_mode);
    if (any) { driven[jt.a] = 1; driven[jt.b] = 1; }
  }
  for (uint32_t i = 0; i < count; ++i) {
    if (!dyn[i] || !awake[i]) continue;
    V3 vl = lin[i], va = ang[i];
    Iso old = original[i], pred = predicted[i];
    Iso np{pos[i], rot[i]};
    // split impulse only outside articulations (step.rs:324-329)
    V3 sl = jointed[i] ? V3{0, 0, 0} : split_l[i], sa = jointed[i] ? V3{0, 0, 0} : split_a[i];
    V3 d_lin = sub(sub(np.pos, pred.pos), sl);
    if (!vzero(d_lin)) vl = add(vl, divs(d_lin, dt));
    if (touching[i] && vl.y < 0.0f) {
      vl.y = 0.0f;
      np.pos.y = old.pos.y;
      set_pose(i, np);
    }
    if (!driven[i] && !qeq(np.rot, pred.rot)) {
      Q4 dq = qmul(np.rot, qconj(pred.rot));
      V3 d_ang = mul(V3{dq.x, dq.y, dq.z}, 2.0f);
      if (dq.w < 0.0f) d_ang = neg(d_ang);
      va = add(va, divs(sub(d_ang, sa), dt));
    }
    set_vel(i, vl, va);
  }
  for (uint32_t i = 0; i < count; ++i) last_lin_vel[i] = lin[i];
  // --- Stage 7: sleep (sleep.rs:59-80), AABBs, contacts kept
  for (uint32_t i = 0; i < count; ++i) {
    if (!sleep_allowed[i]) continue;
    if (!awake[i] || !dyn[i]) continue;
    if (len2(lin[i]) < 0.01f && len2(ang[i]) < 0.01f) {
      sleep_ticks[i] = (uint16_t)(sleep_ticks[i] + 1);
      if (sleep_ticks[i] > 30) awake[i] = 0;
    } else {
      sleep_ticks[i] = 0;
    }
  }
  update_colliders_aabb();
  last_frame_contacts = contacts;
  last_levels = levels_out;
}

// World::step_hash (provenance.rs:6-24) + hash_carried (world.rs:882-909)
void World::step_hash(uint8_t out[32]) const {
  b3::Hasher h;
  h.update_u64(epoch);
  h.update_u64(rng);
  static const uint8_t kEmptyDigest[32] = {
      0xaf, 0x13, 0x49, 0xb9, 0xf5, 0xf9, 0xa1, 0xa6, 0xa0, 0x40, 0x4d, 0xea, 0x36, 0xdc, 0xc9, 0x49,
      0x9b, 0xcb, 0x25, 0xc9, 0xad, 0xc1, 0x12, 0xb7, 0xcc, 0x9a, 0x93, 0xca, 0xe4, 0x1f, 0x32, 0x62};
  h.update(kEmptyDigest, 32);  // ScheduleRecorder::digest of no stages = BLAKE3("")
  auto v3h = [&](V3 v) { h.update_u32(canon_bits(v.x)); h.update_u32(canon_bits(v.y)); h.update_u32(canon_bits(v.z)); };
  for (uint32_t i = 0; i < num_bodies(); ++i) {
    h.update_u32(i);
    v3h(pos[i]);
    h.update_u32(canon_bits(rot[i].x)); h.update_u32(canon_bits(rot[i].y));
    h.update_u32(canon_bits(rot[i].z)); h.update_u32(canon_bits(rot[i].w));
    v3h(lin[i]);
    v3h(ang[i]);
  }
  h.update_u64(warm.size());
  for (auto& kv : warm) {
    h.update_u32(std::get<0>(kv.first)); h.update_u32(std::get<1>(kv.first));
    h.update_u32(std::get<2>(kv.first)); h.update_u32(std::get<3>(kv.first));
    h.update_u32((uint32_t)kv.second.size());
    for (auto& c : kv.second) { v3h(c.la); h.update_u32(canon_bits(c.jn)); v3h(c.jt); }
  }
  h.update_u64(0);  // warm_patches
  h.update_u64(warm_joints.size());
  for (auto& kv : warm_joints) {
    h.update_u32(kv.first);
    h.update_u32((uint32_t)kv.second.size());
    for (auto& r : kv.second) { h.update_u8(r.first); h.update_u32(canon_bits(r.second)); }
  }
  h.update_u64(0);  // rotor
  h.update_u64(last_lin_vel.size());
  for (auto& v : last_lin_vel) v3h(v);
  h.update_u64(awake.size());
  for (auto a : awake) h.update_u8(a);
  h.update_u64(sleep_ticks.size());
  for (auto t : sleep_ticks) { uint8_t b[2] = {(uint8_t)t, (uint8_t)(t >> 8)}; h.update(b, 2); }
  h.finalize(out);
}

}  // namespace orc
