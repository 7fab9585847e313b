// rp_narrow.cuh -- device narrowphase: one thread computes one shape pair's contact manifold
// (at most 4 points, fixed slots), following riftphys-collision/src/narrowphase.rs:
//   collide_shapes dispatch (:73-161), box-box SAT + incident-face clipping + reduce_to_4
//   (:173-338), box-triangle (:349-409), sphere-sphere (:412-442), capsule pairs (:444-537),
//   box-sphere / box-capsule (:540-622), triangle routines (:627-733).
// Clipping polygons (<= 8 vertices) and the candidate lists live in registers/local memory.
#pragma once
#include "rp_math.cuh"

namespace rp {

struct Shape { uint32_t kind; float a, b, c; };
struct Tri { f3 a, b, c; };
struct Iso { f3 pos; q4 rot; };
struct CP { f3 position, normal; float penetration; };
struct Manifold { f3 normal; CP pts[4]; int len; };

__device__ __forceinline__ void mpush(Manifold* m, const CP& p) { if (m->len < 4) m->pts[m->len++] = p; }
__device__ __forceinline__ f3 norm_or(f3 v, f3 fb) {
  v = fin_v(v);
  float l2 = len2(v);
  if (l2 > 1.0e-12f) return v * (1.0f / sqrtf(l2));
  return fb;
}
__device__ __forceinline__ void mflip(Manifold* m) {
  m->normal = -m->normal;
  for (int i = 0; i < m->len; ++i) m->pts[i].normal = m->normal;
}

// reduce_to_4 (:312-338). Candidates in arrays; writes up to 4 indices.
__device__ __forceinline__ int reduce_to_4(const float* dep, const f3* pt, int n, f3 nrm, int* out) {
  if (n <= 4) { for (int i = 0; i < n; ++i) out[i] = i; return n; }
  int cnt = 0;
  // argmax by sort_key6, lowest index on ties
  int i0 = 0; long long k0 = LLONG_MIN;
  for (int i = 0; i < n; ++i) { long long k = sort_key6(dep[i]); if (k > k0) { k0 = k; i0 = i; } }
  f3 p0 = pt[i0];
  out[cnt++] = i0;
  int i1 = 0; long long k1 = LLONG_MIN; float d1 = -INFINITY;
  for (int i = 0; i < n; ++i) { float v = len2(pt[i] - p0); long long k = sort_key6(v); if (k > k1) { k1 = k; i1 = i; d1 = v; } }
  if (!(d1 > 1.0e-12f)) return cnt;
  out[cnt++] = i1;
  f3 e = pt[i1] - p0;
  int i2 = 0; long long k2 = LLONG_MIN; float a2 = -INFINITY;
  for (int i = 0; i < n; ++i) {
    float v = fabsf(dot(cross(pt[i] - p0, e), nrm));
    long long k = sort_key6(v);
    if (k > k2) { k2 = k; i2 = i; a2 = v; }
  }
  if (!(a2 > 1.0e-12f)) return cnt;
  out[cnt++] = i2;
  float s2 = signum(dot(cross(pt[i2] - p0, e), nrm));
  int i3 = 0; long long k3 = LLONG_MIN; float a3 = -INFINITY;
  for (int i = 0; i < n; ++i) {
    float v = -dot(cross(pt[i] - p0, e), nrm) * s2;
    long long k = sort_key6(v);
    if (k > k3) { k3 = k; i3 = i; a3 = v; }
  }
  if (a3 > 1.0e-12f) out[cnt++] = i3;
  return cnt;
}

// clip_poly (:289-301): keeps p.n <= d
__device__ __forceinline__ int clip_poly(const f3* in, int n, f3 nn, float d, f3* out) {
  int m = 0;
  for (int i = 0; i < n; ++i) {
    f3 p = in[i], q = in[(i + 1) % n];
    float dp = dot(p, nn) - d, dq = dot(q, nn) - d;
    if (dp <= 0.0f) out[m++] = p;
    if ((dp <= 0.0f) != (dq <= 0.0f)) {
      float t = dp / (dp - dq);
      out[m++] = p + (q - p) * t;
    }
  }
  return m;
}
__device__ __forceinline__ float radius3(const f3* ax, const float* e, f3 l) {
  return (e[0] * fabsf(dot(ax[0], l)) + e[1] * fabsf(dot(ax[1], l))) + e[2] * fabsf(dot(ax[2], l));
}

// collide_box_box (:173-256) with clip_incident_face (:261-286)
static __device__ bool box_box(const Iso& xa, f3 ea, const Iso& xb, f3 eb, float cd, Manifold* m) {
  f3 aa[3] = {qrot(xa.rot, mk3(1, 0, 0)), qrot(xa.rot, mk3(0, 1, 0)), qrot(xa.rot, mk3(0, 0, 1))};
  f3 ba[3] = {qrot(xb.rot, mk3(1, 0, 0)), qrot(xb.rot, mk3(0, 1, 0)), qrot(xb.rot, mk3(0, 0, 1))};
  float ear[3] = {ea.x, ea.y, ea.z}, ebr[3] = {eb.x, eb.y, eb.z};
  f3 t = xb.pos - xa.pos;
  bool have = false; float bo = 0.0f; f3 bl = mk3(0, 0, 0); int bw = 0;
  for (int k = 0; k < 15; ++k) {
    f3 l; int which;
    if (k < 3) { l = aa[k]; which = k; }
    else if (k < 6) { l = ba[k - 3]; which = k; }
    else { int i = (k - 6) / 3, j = (k - 6) % 3; l = cross(aa[i], ba[j]); which = 6; }
    float l2 = len2(l);
    if (l2 < 1.0e-10f) continue;
    l = l / sqrtf(l2);
    float overlap = (radius3(aa, ear, l) + radius3(ba, ebr, l)) - fabsf(dot(t, l));
    if (overlap < -cd) return false;
    bool is_face = which < 6;
    bool better;
    if (!have) better = true;
    else {
      bool face = bw < 6;
      if (is_face && face && ((which >= 3) != (bw >= 3))) better = overlap < bo - (0.02f * fabsf(bo) + 1.0e-3f);
      else if (is_face == face) better = overlap < bo;
      else if (is_face) better = overlap < bo * 1.05f + 1.0e-4f;
      else better = overlap < bo * 0.95f - 1.0e-4f;
    }
    if (better) { have = true; bo = overlap; bl = l; bw = which; }
  }
  if (!have) return false;
  f3 n = dot(t, bl) < 0.0f ? -bl : bl;
  f3 normal = norm_or(n, mk3(0, 1, 0));
  m->normal = normal; m->len = 0;
  if (bw == 6) {
    f3 sa = xa.pos + normal * radius3(aa, ear, normal);
    f3 sb = xb.pos - normal * radius3(ba, ebr, normal);
    CP c; c.position = fin_v((sa + sb) * 0.5f); c.normal = normal; c.penetration = fin0(bo + cd);
    mpush(m, c);
    return true;
  }
  // reference / incident selection
  bool ref_a = bw < 3;
  f3 rc = ref_a ? xa.pos : xb.pos, ic = ref_a ? xb.pos : xa.pos;
  const float* re = ref_a ? ear : ebr;
  const float* ie = ref_a ? ebr : ear;
  const f3* rax = ref_a ? aa : ba;
  const f3* iax = ref_a ? ba : aa;
  int k = ref_a ? bw : bw - 3;
  f3 nr = ref_a ? normal : -normal;
  // clip_incident_face
  int f = 0; float fd = -INFINITY;
  for (int i = 0; i < 3; ++i) { float d = fabsf(dot(iax[i], nr)); if (d > fd) { fd = d; f = i; } }
  float s = dot(iax[f], nr) > 0.0f ? -1.0f : 1.0f;
  int u = (f + 1) % 3, v = (f + 2) % 3;
  f3 c = ic + iax[f] * (s * ie[f]);
  f3 du = iax[u] * ie[u], dv = iax[v] * ie[v];
  f3 pa[9], pb[9];
  pa[0] = (c + du) + dv; pa[1] = (c - du) + dv; pa[2] = (c - du) - dv; pa[3] = (c + du) - dv;
  int np = 4;
  for (int jj = 0; jj < 2 && np > 0; ++jj) {
    int j = (k + 1 + jj) % 3;
    f3 ax = rax[j];
    float mid = dot(rc, ax);
    np = clip_poly(pa, np, ax, mid + re[j], pb);
    if (np == 0) break;
    np = clip_poly(pb, np, -ax, -(mid - re[j]), pa);
  }
  float cdep[9]; f3 cpt[9]; int nc = 0;
  if (np > 0) {
    float plane = dot(rc, nr) + re[k];
    for (int i = 0; i < np; ++i) {
      float depth = plane - dot(pa[i], nr);
      if (depth > -cd) { cdep[nc] = depth; cpt[nc] = pa[i] + nr * (0.5f * depth); nc++; }
    }
  }
  if (nc == 0) {
    f3 sa = xa.pos + normal * radius3(aa, ear, normal);
    f3 sb = xb.pos - normal * radius3(ba, ebr, normal);
    CP cc; cc.position = fin_v((sa + sb) * 0.5f); cc.normal = normal; cc.penetration = fin0(bo + cd);
    mpush(m, cc);
    return true;
  }
  int idx[4];
  int r = reduce_to_4(cdep, cpt, nc, normal, idx);
  for (int i = 0; i < r; ++i) {
    CP cc; cc.position = fin_v(cpt[idx[i]]); cc.normal = normal; cc.penetration = fin0(cdep[idx[i]] + cd);
    mpush(m, cc);
  }
  return true;
}

__device__ __forceinline__ bool sphere_sphere(f3 ca, float ra, f3 cb, float rb, float cd, Manifold* m) {
  f3 delta = cb - ca;
  float d2 = len2(delta);
  ra = fin0(rmax(ra, 0.0f)); rb = fin0(rmax(rb, 0.0f));
  float allowed = fin0((ra + rb) + cd);
  if (!fin(d2) || d2 > allowed * allowed) return false;
  float dist = sqrtf(d2);
  f3 raw = dist > 1.0e-6f ? delta / dist : mk3(1, 0, 0);
  f3 normal = norm_or(raw, mk3(1, 0, 0));
  float pen = fin0(rmax(allowed - dist, 0.0f));
  f3 pa = ca + normal * ra, pb = cb - normal * rb;
  m->normal = normal; m->len = 0;
  CP c; c.position = fin_v((pa + pb) * 0.5f); c.normal = normal; c.penetration = pen;
  mpush(m, c);
  return true;
}
__device__ __forceinline__ void capsule_segment(const Iso& xf, float half, f3* a, f3* b) {
  f3 axis = qrot(xf.rot, mk3(0, 1, 0));
  float h = fabsf(half);
  *a = xf.pos - axis * h;
  *b = xf.pos + axis * h;
}
__device__ __forceinline__ f3 closest_point_segment(f3 p, f3 a, f3 b) {
  f3 ab = b - a;
  float l2 = len2(ab);
  if (l2 <= 1.0e-12f) return a;
  float t = clampf(dot(p - a, ab) / l2, 0.0f, 1.0f);
  return a + ab * t;
}
__device__ __forceinline__ void closest_seg_seg(f3 p0, f3 p1, f3 q0, f3 q1, f3* ra, f3* rb) {
  f3 u = p1 - p0, v = q1 - q0, w = p0 - q0;
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
    if (-d < 0.0f) sn = 0.0f; else if (-d > a) sn = sd; else { sn = -d; sd = a; }
  } else if (tn > td) {
    tn = td;
    if ((-d + b) < 0.0f) sn = 0.0f; else if ((-d + b) > a) sn = sd; else { sn = -d + b; sd = a; }
  }
  float sc = fabsf(sn) < EPS ? 0.0f : sn / sd;
  float tc = fabsf(tn) < EPS ? 0.0f : tn / td;
  *ra = p0 + u * sc;
  *rb = q0 + v * tc;
}
__device__ __forceinline__ bool box_sphere(const Iso& bx, f3 e, f3 sc, float sr, float cd, Manifold* m) {
  f3 pl = fin_v(qrot(qconj(bx.rot), sc - bx.pos));
  f3 cl = mk3(rmin(rmax(pl.x, -e.x), e.x), rmin(rmax(pl.y, -e.y), e.y), rmin(rmax(pl.z, -e.z), e.z));
  float r = fin0(rmax(sr, 0.0f));
  float allowed = fin0(r + cd);
  f3 yw = qrot(bx.rot, mk3(0, 1, 0));
  if (veq(cl, pl)) {
    f3 dtf = e - vabs(pl);
    f3 axis; float depth;
    if (dtf.x < dtf.y && dtf.x < dtf.z) { axis = mk3(1, 0, 0) * (pl.x > 0.0f ? 1.0f : -1.0f); depth = dtf.x; }
    else if (dtf.y < dtf.z) { axis = mk3(0, 1, 0) * (pl.y > 0.0f ? 1.0f : -1.0f); depth = dtf.y; }
    else { axis = mk3(0, 0, 1) * (pl.z > 0.0f ? 1.0f : -1.0f); depth = dtf.z; }
    f3 normal = norm_or(qrot(bx.rot, axis), yw);
    f3 face = fin_v(sc + normal * depth);
    CP c; c.position = fin_v((face + (sc - normal * r)) * 0.5f); c.normal = normal;
    c.penetration = fin0(allowed + rmax(depth, 0.0f));
    m->normal = normal; m->len = 0;
    mpush(m, c);
    return true;
  }
  f3 cw = fin_v(bx.pos + qrot(bx.rot, cl));
  f3 delta = sc - cw;
  float dist = sqrtf(len2(delta));
  if (dist > allowed) return false;
  f3 raw = dist > 1.0e-6f ? delta / dist : yw;
  f3 normal = norm_or(raw, yw);
  CP c; c.position = fin_v((cw + (sc - normal * r)) * 0.5f); c.normal = normal; c.penetration = fin0(allowed - dist);
  m->normal = normal; m->len = 0;
  mpush(m, c);
  return true;
}
__device__ __forceinline__ bool box_capsule(const Iso& bx, f3 e, const Iso& cx, float cr, float ch, float cd, Manifold* m) {
  f3 aw, bw; capsule_segment(cx, ch, &aw, &bw);
  q4 inv = qconj(bx.rot);
  f3 al = fin_v(qrot(inv, aw - bx.pos));
  f3 bl = fin_v(qrot(inv, bw - bx.pos));
  f3 mid = closest_point_segment(mk3(0, 0, 0), al, bl);
  bool have = false;
  for (int i = 0; i < 3; ++i) {
    f3 p = i == 0 ? al : (i == 1 ? bl : mid);
    f3 pw = bx.pos + qrot(bx.rot, p);
    Manifold t;
    if (box_sphere(bx, e, pw, cr, cd, &t)) {
      if (!have || t.pts[0].penetration > m->pts[0].penetration) { *m = t; have = true; }
    }
  }
  return have;
}
__device__ __forceinline__ f3 closest_point_triangle(f3 p, f3 a, f3 b, f3 c) {
  f3 ab = b - a, ac = c - a, ap = p - a;
  float d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) return a;
  f3 bp = p - b;
  float d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) return b;
  float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) { float v = d1 / (d1 - d3); return a + ab * v; }
  f3 cp = p - c;
  float d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) return c;
  float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) { float w = d2 / (d2 - d6); return a + ac * w; }
  float va = d3 * d6 - d5 * d4;
  if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
    float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return b + (c - b) * w;
  }
  float denom = 1.0f / ((va + vb) + vc);
  float v = vb * denom, w = vc * denom;
  return (a + ab * v) + ac * w;
}
// Triangle vertices through the identity transform the terrain query attaches (Isometry::IDENTITY)
__device__ __forceinline__ void tri_world(const Tri& t, f3* a, f3* b, f3* c) {
  f3 z = mk3(0, 0, 0);
  *a = z + qrot(qident(), t.a); *b = z + qrot(qident(), t.b); *c = z + qrot(qident(), t.c);
}
__device__ __forceinline__ bool sphere_triangle(f3 sc, float sr, const Tri& tri, float cd, Manifold* m) {
  f3 a, b, c; tri_world(tri, &a, &b, &c);
  f3 cl = closest_point_triangle(sc, a, b, c);
  f3 delta = sc - cl;
  float d2 = len2(delta);
  float r = fin0(rmax(sr, 0.0f));
  float allowed = fin0(r + cd);
  if (d2 > allowed * allowed) return false;
  float dist = sqrtf(d2);
  f3 tn = normalize_or_zero(cross(b - a, c - a));
  f3 raw = dist > 1.0e-6f ? delta / dist : tn;
  f3 normal = norm_or(raw, tn);
  m->normal = normal; m->len = 0;
  CP cc; cc.position = fin_v(cl); cc.normal = normal; cc.penetration = fin0(allowed - dist);
  mpush(m, cc);
  return true;
}
__device__ __forceinline__ bool capsule_triangle(const Iso& cx, float cr, float ch, const Tri& tri, float cd, Manifold* m) {
  f3 aw, bw; capsule_segment(cx, ch, &aw, &bw);
  f3 mid = (aw + bw) * 0.5f;
  bool have = false;
  for (int i = 0; i < 3; ++i) {
    f3 p = i == 0 ? aw : (i == 1 ? bw : mid);
    Manifold t;
    if (sphere_triangle(p, cr, tri, cd, &t)) {
      if (!have || t.pts[0].penetration > m->pts[0].penetration) { *m = t; have = true; }
    }
  }
  return have;
}
static __device__ bool box_triangle(const Iso& bx, f3 e, const Tri& tri, float cd, Manifold* m) {
  f3 ta, tb, tc; tri_world(tri, &ta, &tb, &tc);
  f3 raw = cross(tb - ta, tc - ta);
  if (!(len2(raw) > 1.0e-12f) || !vfin(raw)) return false;
  f3 n = normalize(raw);
  f3 ax[3] = {qrot(bx.rot, mk3(1, 0, 0)), qrot(bx.rot, mk3(0, 1, 0)), qrot(bx.rot, mk3(0, 0, 1))};
  float er[3] = {e.x, e.y, e.z};
  float r = radius3(ax, er, n);
  float centre = dot(bx.pos - ta, n);
  if (centre - r > cd) return false;
  int f = 0; float fd = -INFINITY;
  for (int i = 0; i < 3; ++i) { float d = fabsf(dot(ax[i], n)); if (d > fd) { fd = d; f = i; } }
  float sgn = dot(ax[f], n) > 0.0f ? -1.0f : 1.0f;
  int u = (f + 1) % 3, v = (f + 2) % 3;
  f3 c = bx.pos + ax[f] * (sgn * er[f]);
  f3 du = ax[u] * er[u], dv = ax[v] * er[v];
  f3 pa[8], pb[8];
  pa[0] = (c + du) + dv; pa[1] = (c - du) + dv; pa[2] = (c - du) - dv; pa[3] = (c + du) - dv;
  int np = 4;
  for (int k = 0; k < 3; ++k) {
    f3 p = k == 0 ? ta : (k == 1 ? tb : tc);
    f3 q = k == 0 ? tb : (k == 1 ? tc : ta);
    f3 out = cross(q - p, n);
    if (!(len2(out) > 1.0e-12f)) return false;
    out = normalize(out);
    np = clip_poly(pa, np, out, dot(p, out), pb);
    if (np == 0) return false;
    for (int i = 0; i < np; ++i) pa[i] = pb[i];
  }
  float cdep[8]; f3 cpt[8]; int nc = 0;
  for (int i = 0; i < np; ++i) {
    float dist = dot(pa[i] - ta, n);
    if (dist <= cd) { cdep[nc] = -dist; cpt[nc] = pa[i] - n * (0.5f * dist); nc++; }
  }
  if (nc == 0) return false;
  f3 normal = -n;
  m->normal = normal; m->len = 0;
  int idx[4];
  int rr = reduce_to_4(cdep, cpt, nc, normal, idx);
  for (int i = 0; i < rr; ++i) {
    CP cc; cc.position = fin_v(cpt[idx[i]]); cc.normal = normal; cc.penetration = fin0(cd + cdep[idx[i]]);
    mpush(m, cc);
  }
  return true;
}

// collide_shapes (:73-161) for collider pairs (no triangles)
static __device__ bool collide_pair(const Shape& a, const Iso& xa, const Shape& b, const Iso& xb, float cd, Manifold* m) {
  m->len = 0;
  if (!vfin(xa.pos) || !vfin(xb.pos)) return false;
  cd = fin0(rmax(cd, 0.0f));
  uint32_t ka = a.kind, kb = b.kind;
  bool ok = false;
  if (ka == SH_SPHERE && kb == SH_SPHERE) ok = sphere_sphere(xa.pos, a.a, xb.pos, b.a, cd, m);
  else if (ka == SH_CAPSULE && kb == SH_SPHERE) { f3 p, q; capsule_segment(xa, a.b, &p, &q); ok = sphere_sphere(closest_point_segment(xb.pos, p, q), a.a, xb.pos, b.a, cd, m); }
  else if (ka == SH_SPHERE && kb == SH_CAPSULE) { f3 p, q; capsule_segment(xb, b.b, &p, &q); ok = sphere_sphere(closest_point_segment(xa.pos, p, q), b.a, xa.pos, a.a, cd, m); if (ok) mflip(m); }
  else if (ka == SH_CAPSULE && kb == SH_CAPSULE) {
    f3 a0, a1, b0, b1; capsule_segment(xa, a.b, &a0, &a1); capsule_segment(xb, b.b, &b0, &b1);
    f3 pa, pb; closest_seg_seg(a0, a1, b0, b1, &pa, &pb);
    ok = sphere_sphere(pa, a.a, pb, b.a, cd, m);
  }
  else if (ka == SH_BOX && kb == SH_SPHERE) ok = box_sphere(xa, mk3(a.a, a.b, a.c), xb.pos, b.a, cd, m);
  else if (ka == SH_SPHERE && kb == SH_BOX) { ok = box_sphere(xb, mk3(b.a, b.b, b.c), xa.pos, a.a, cd, m); if (ok) mflip(m); }
  else if (ka == SH_BOX && kb == SH_CAPSULE) ok = box_capsule(xa, mk3(a.a, a.b, a.c), xb, b.a, b.b, cd, m);
  else if (ka == SH_CAPSULE && kb == SH_BOX) { ok = box_capsule(xb, mk3(b.a, b.b, b.c), xa, a.a, a.b, cd, m); if (ok) mflip(m); }
  else if (ka == SH_BOX && kb == SH_BOX) ok = box_box(xa, mk3(a.a, a.b, a.c), xb, mk3(b.a, b.b, b.c), cd, m);
  if (!ok) m->len = 0;
  return ok;
}
// collide_shapes for a collider against one terrain triangle
static __device__ bool collide_tri(const Shape& a, const Iso& xa, const Tri& t, float cd, Manifold* m) {
  m->len = 0;
  if (!vfin(xa.pos)) return false;
  cd = fin0(rmax(cd, 0.0f));
  bool ok = false;
  if (a.kind == SH_SPHERE) ok = sphere_triangle(xa.pos, a.a, t, cd, m);
  else if (a.kind == SH_CAPSULE) ok = capsule_triangle(xa, a.a, a.b, t, cd, m);
  else if (a.kind == SH_BOX) ok = box_triangle(xa, mk3(a.a, a.b, a.c), t, cd, m);
  if (!ok) m->len = 0;
  return ok;
}

}  // namespace rp
