// query.cu -- ray casts on the device (riftphys-world/src/world/queries.rs:50-116): against every
// collider's stored AABB (geom.rs:40-93), then against the heightfield's triangles in the ray's
// box (terrain.rs:300-358, triangle.rs:215-235). One block per ray: its threads test a chunk of
// colliders (or triangles) at once, then one thread takes the chunk's hits in index order with
// the reference's replacement rule, so the result is the sequential scan's exactly.
#include "hf_cells.cuh"
#include "rp_narrow.cuh"
#include "shape_aabb.cuh"
#include "step_internal.cuh"

namespace rp {

namespace {
constexpr int QT = 256;  // threads per ray
}

struct RayIn { f3 o, d; float max_d; uint32_t ignore; };  // d normalised; ignore: body index or kNoBody
constexpr uint32_t kNoBody = 0xFFFFFFFFu;
static_assert(sizeof(RayIn) == 32, "RayIn: 8 words per ray");

// normal_from_aabb_point (geom.rs:40-57)
__device__ f3 normal_from_aabb_point(f3 mn, f3 mx, f3 p) {
  const float eps = 1.0e-4f;
  if (fabsf(p.x - mn.x) < eps) return mk3(-1, 0, 0);
  if (fabsf(p.x - mx.x) < eps) return mk3(1, 0, 0);
  if (fabsf(p.y - mn.y) < eps) return mk3(0, -1, 0);
  if (fabsf(p.y - mx.y) < eps) return mk3(0, 1, 0);
  if (fabsf(p.z - mn.z) < eps) return mk3(0, 0, -1);
  if (fabsf(p.z - mx.z) < eps) return mk3(0, 0, 1);
  f3 c = (mn + mx) * 0.5f;
  f3 n = p - c;
  float l2 = len2(n);
  if (l2 > 1.0e-20f) { float l = sqrtf(l2); n = mk3(n.x / l, n.y / l, n.z / l); }
  else n = mk3(0, 1, 0);
  return n;
}
// ray_aabb (geom.rs:59-93): the slab test from t = 0 to max_dist
__device__ bool ray_aabb(f3 o, f3 d, f3 mn, f3 mx, float max_d, float* t_out, f3* p_out, f3* n_out) {
  const float eps = 1.0e-8f;
  float tmin = 0.0f, tmax = max_d;
  const float oo[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z}, lo[3] = {mn.x, mn.y, mn.z}, hi[3] = {mx.x, mx.y, mx.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (fabsf(dd[a]) < eps) {
      if (oo[a] < lo[a] || oo[a] > hi[a]) return false;
    } else {
      float inv = 1.0f / dd[a];
      float t1 = (lo[a] - oo[a]) * inv, t2 = (hi[a] - oo[a]) * inv;
      if (t1 > t2) { float s = t1; t1 = t2; t2 = s; }
      if (t1 > tmin) tmin = t1;
      if (t2 < tmax) tmax = t2;
      if (tmin > tmax) return false;
    }
  }
  if (tmin < 0.0f || tmin > max_d) return false;
  f3 p = o + d * tmin;
  *t_out = tmin;
  *p_out = p;
  *n_out = normal_from_aabb_point(mn, mx, p);
  return true;
}
// Triangle::intersect_ray (triangle.rs:215-235) with Plane::from_points / intersect_ray
// (plane.rs:16-86) and Triangle::barycentric (triangle.rs:74-113); t in [0, max_d].
__device__ bool ray_triangle(f3 o, f3 d, float max_d, f3 a, f3 b, f3 c, float* t_out) {
  f3 n = cross(b - a, c - a);
  float a2 = dot(n, n);
  if (!fin(a2) || a2 <= 1.0e-16f) return false;  // degenerate
  if (!(vfin(a) && vfin(b) && vfin(c))) return false;
  float l2 = dot(n, n);
  if (!fin(l2) || l2 <= 1.0e-6f * 1.0e-6f) return false;
  float inv_len = 1.0f / sqrtf(l2);
  f3 nu = n * inv_len;
  float pd = -dot(nu, a);
  if (!(vfin(nu) && fin(pd))) return false;
  if (!(vfin(o) && vfin(d))) return false;
  float denom = dot(nu, d);
  if (!fin(denom) || fabsf(denom) < 1.0e-6f) return false;
  float numer = -(dot(nu, o) + pd);
  if (!fin(numer)) return false;
  float t = numer / denom;
  if (!fin(t)) return false;
  if (!(t >= 0.0f && t <= max_d)) return false;
  f3 p = o + d * t;
  f3 v0 = b - a, v1 = c - a, v2 = p - a;
  float d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
  float den = d00 * d11 - d01 * d01;
  float scale = rmax(fabsf(d00 * d11), 1.0f);
  if (!fin(den) || fabsf(den) <= 1.0e-12f * scale) return false;
  float inv = 1.0f / den;
  float v = (d11 * d20 - d01 * d21) * inv;
  float w = (d00 * d21 - d01 * d20) * inv;
  float u = 1.0f - v - w;
  if (!(fin(u) && fin(v) && fin(w) && u >= -1.0e-5f && v >= -1.0e-5f && w >= -1.0e-5f)) return false;
  *t_out = t;
  return true;
}
// Triangle::normal (triangle.rs:26-31): normalize_or_zero of the unnormalised normal
__device__ f3 tri_normal(f3 a, f3 b, f3 c) {
  f3 n = cross(b - a, c - a);
  if (!vfin(n)) return mk3(0, 0, 0);
  float rcp = 1.0f / sqrtf(dot(n, n));
  return (fin(rcp) && rcp > 0.0f) ? n * rcp : mk3(0, 0, 0);
}

__global__ void __launch_bounds__(QT) k_raycast(uint32_t nrays, const RayIn* __restrict__ rays, uint32_t ncol,
                                                const uint32_t* __restrict__ cbody, const uint32_t* __restrict__ ckind,
                                                const float4* __restrict__ cdims, const float4* __restrict__ pos,
                                                const float4* __restrict__ rot, const uint8_t* __restrict__ alive,
                                                bool has_hf, HfDev hf, float4* out_pt, float4* out_n) {
  const uint32_t r = blockIdx.x;
  if (r >= nrays) return;
  const int tid = threadIdx.x;
  const RayIn ray = rays[r];
  __shared__ float s_t[QT];
  __shared__ float4 s_p[QT], s_n[QT];
  __shared__ uint8_t s_hit[QT];
  __shared__ float b_t;
  __shared__ uint32_t b_ci;
  __shared__ f3 b_p, b_n;
  __shared__ int have;
  if (tid == 0) { have = 0; b_t = 0.0f; b_ci = 0; }
  __syncthreads();
  // 1. colliders, in index order: take a hit when it is the first, or nearer by more than 1e-9
  //    (or as near and of a lower index, which a scan in index order never sees)
  for (uint32_t base = 0; base < ncol; base += QT) {
    const uint32_t ci = base + tid;
    bool hit = false;
    if (ci < ncol) {
      const uint32_t bd = cbody[ci];
      if (alive[bd] && bd != ray.ignore) {
        f3 mn, mx;
        aabb_of(ckind[ci], cdims[ci], xyz(pos[bd]), asq(rot[bd]), &mn, &mx);
        float t;
        f3 p, n;
        hit = ray_aabb(ray.o, ray.d, mn, mx, ray.max_d, &t, &p, &n);
        if (hit) { s_t[tid] = t; s_p[tid] = f4(p); s_n[tid] = f4(n); }
      }
    }
    s_hit[tid] = hit ? 1 : 0;
    __syncthreads();
    if (tid == 0) {
      for (int k = 0; k < QT; ++k) {
        if (!s_hit[k]) continue;
        const float t = s_t[k];
        const uint32_t ci2 = base + k;
        if (!have || (t < b_t - 1.0e-9f) || (fabsf(t - b_t) <= 1.0e-9f && ci2 < b_ci)) {
          have = 1; b_t = t; b_ci = ci2; b_p = xyz(s_p[k]); b_n = xyz(s_n[k]);
        }
      }
    }
    __syncthreads();
  }
  // 2. the heightfield's triangles in the ray's box, cell by cell: nearer by more than 1e-9 wins
  if (has_hf) {
    const f3 end = ray.o + ray.d * ray.max_d;
    f3 qa = vmin(ray.o, end), qb = vmax(ray.o, end);
    qa = mk3(qf32(qa.x), qf32(qa.y), qf32(qa.z));
    qb = mk3(qf32(qb.x), qf32(qb.y), qf32(qb.z));
    const f3 qmn = vmin(qa, qb), qmx = vmax(qa, qb);
    const int nx = (int)hf.nx, nz = (int)hf.nz;
    if (nx >= 2 && nz >= 2 && !(qmn.y > hf.max_y + 1.0f || qmx.y < hf.min_y - 1.0f)) {
      auto toi = [](float f) -> long long {
        if (isnan(f)) return 0;
        if (f >= 2147483647.0f) return 2147483647;
        if (f <= -2147483648.0f) return -2147483648LL;
        return (long long)f;
      };
      auto cl = [](long long v, long long lo, long long hi) { return v < lo ? lo : (v > hi ? hi : v); };
      const long long gx0 = cl(toi(floorf((qmn.x - hf.ox) / hf.sx)) - 1, 0, nx - 2);
      const long long gx1 = cl(toi(ceilf((qmx.x - hf.ox) / hf.sx)) + 1, 0, nx - 2);
      const long long gz0 = cl(toi(floorf((qmn.z - hf.oz) / hf.sz)) - 1, 0, nz - 2);
      const long long gz1 = cl(toi(ceilf((qmx.z - hf.oz) / hf.sz)) + 1, 0, nz - 2);
      const unsigned long long wx = (unsigned long long)(gx1 - gx0 + 1), ntri = 2ull * wx * (unsigned long long)(gz1 - gz0 + 1);
      for (unsigned long long base = 0; base < ntri; base += QT) {
        const unsigned long long k = base + tid;
        bool hit = false;
        if (k < ntri) {
          const unsigned long long cell = k >> 1;
          const long long gz = gz0 + (long long)(cell / wx), gx = gx0 + (long long)(cell % wx);
          auto H = [&](long long x, long long z) { return hf.h[(size_t)x + (size_t)z * hf.nx]; };
          const float x0 = (float)gx * hf.sx + hf.ox, x1 = x0 + hf.sx;
          const float z0 = (float)gz * hf.sz + hf.oz, z1 = z0 + hf.sz;
          const f3 p00 = mk3(x0, H(gx, gz), z0), p10 = mk3(x1, H(gx + 1, gz), z0);
          const f3 p01 = mk3(x0, H(gx, gz + 1), z1), p11 = mk3(x1, H(gx + 1, gz + 1), z1);
          f3 a = p00, b = p01, c = p10;  // tri1 = (p00, p01, p10), tri2 = (p10, p01, p11)
          if (k & 1ull) { a = p10; b = p01; c = p11; }
          float t;
          hit = ray_triangle(ray.o, ray.d, ray.max_d, a, b, c, &t);
          if (hit) {
            s_t[tid] = t;
            s_p[tid] = f4(ray.o + ray.d * t);
            s_n[tid] = f4(tri_normal(a, b, c));
          }
        }
        s_hit[tid] = hit ? 1 : 0;
        __syncthreads();
        if (tid == 0) {
          for (int q = 0; q < QT; ++q) {
            if (!s_hit[q]) continue;
            const float t = s_t[q];
            if (!have || t < b_t - 1.0e-9f) { have = 1; b_t = t; b_ci = kNoBody; b_p = xyz(s_p[q]); b_n = xyz(s_n[q]); }
          }
        }
        __syncthreads();
      }
    }
  }
  if (tid == 0) {
    if (!have) {
      out_pt[r] = make_float4(0, 0, 0, __uint_as_float(0u));
      out_n[r] = make_float4(0, 1, 0, 1.0f);
    } else {
      const uint32_t body = b_ci == kNoBody ? kNoBody : cbody[b_ci];
      out_pt[r] = make_float4(b_p.x, b_p.y, b_p.z, __uint_as_float(body == kNoBody ? kNoBody : body + 1u));
      out_n[r] = make_float4(b_n.x, b_n.y, b_n.z, clampf(b_t / ray.max_d, 0.0f, 1.0f));
    }
  }
}

// ---- capsule sweeps (queries.rs:118-249): a y-axis capsule at from, overlap at t = 0 first, then
// its tip and base spheres swept along to - from against the colliders' and the terrain
// triangles' AABBs (riftphys-query/src/lib.rs:1-134).
struct SweepIn { f3 from, to; float r, hh; uint32_t ignore; uint32_t pad[3]; };
static_assert(sizeof(SweepIn) == 48, "SweepIn: 12 words per sweep");
constexpr float kToiEps = 1e-9f;  // TOI_EPS (lib.rs:4) and the sweep's eps (queries.rs:185)
// ray_aabb_slab_unit (lib.rs:42-79)
__device__ bool ray_aabb_slab_unit(f3 o, f3 d, f3 mn, f3 mx, float* t_out, f3* n_out) {
  const f3 inv = mk3((o.x == o.x && fabsf(d.x) > 1e-9f) ? 1.0f / d.x : 1.0e9f,
                     (o.y == o.y && fabsf(d.y) > 1e-9f) ? 1.0f / d.y : 1.0e9f,
                     (o.z == o.z && fabsf(d.z) > 1e-9f) ? 1.0f / d.z : 1.0e9f);
  const f3 t1 = mk3((mn.x - o.x) * inv.x, (mn.y - o.y) * inv.y, (mn.z - o.z) * inv.z);
  const f3 t2 = mk3((mx.x - o.x) * inv.x, (mx.y - o.y) * inv.y, (mx.z - o.z) * inv.z);
  const f3 tmin = vmin(t1, t2), tmax = vmax(t1, t2);
  float t_enter = tmin.x;
  f3 n = mk3(t1.x > t2.x ? 1.0f : -1.0f, 0.0f, 0.0f);
  if (tmin.y > t_enter) { t_enter = tmin.y; n = mk3(0.0f, t1.y > t2.y ? 1.0f : -1.0f, 0.0f); }
  if (tmin.z > t_enter) { t_enter = tmin.z; n = mk3(0.0f, 0.0f, t1.z > t2.z ? 1.0f : -1.0f); }
  const float t_exit = rmin(rmin(tmax.x, tmax.y), tmax.z);
  if (t_enter <= t_exit && t_exit >= 0.0f && t_enter >= 0.0f && t_enter <= 1.0f) { *t_out = t_enter; *n_out = n; return true; }
  return false;
}
// sweep_sphere_aabb (lib.rs:81-104) with dt = 1
__device__ bool sweep_sphere_aabb(f3 p0, f3 v, float r, f3 mn, f3 mx, float* t, f3* n) {
  const f3 dir = v * 1.0f;
  const f3 e = splat(r);
  const f3 emn = mn - e, emx = mx + e;
  if (len2(dir) < 1e-12f) {
    const bool inside = p0.x >= emn.x && p0.x <= emx.x && p0.y >= emn.y && p0.y <= emx.y && p0.z >= emn.z && p0.z <= emx.z;
    if (inside) { *t = 0.0f; *n = mk3(0, 1, 0); }
    return inside;
  }
  return ray_aabb_slab_unit(p0, dir, emn, emx, t, n);
}
// sweep_two_spheres_aabbs for one AABB (lib.rs:118-134): the tip's hit, then the base's, by pick_better
__device__ bool sweep_two(f3 tip0, f3 base0, f3 v, float r, f3 mn, f3 mx, float* t, f3* n, int* kind) {
  bool have = false;
  float tt;
  f3 nn;
  if (sweep_sphere_aabb(tip0, v, r, mn, mx, &tt, &nn)) { have = true; *t = tt; *n = nn; *kind = 0; }
  if (sweep_sphere_aabb(base0, v, r, mn, mx, &tt, &nn)) {
    // pick_better: nearer by more than TOI_EPS, or as near with the same target and a lower kind
    // (never: the base is kind 1)
    if (!have || tt < *t - kToiEps) { have = true; *t = tt; *n = nn; *kind = 1; }
  }
  return have;
}

__global__ void __launch_bounds__(QT) k_sweep(uint32_t nq, const SweepIn* __restrict__ qs, uint32_t ncol,
                                              const uint32_t* __restrict__ cbody, const uint32_t* __restrict__ ckind,
                                              const float4* __restrict__ cdims, const float4* __restrict__ pos,
                                              const float4* __restrict__ rot, const uint8_t* __restrict__ alive,
                                              bool has_hf, HfDev hf, float4* out_pt, float4* out_n) {
  const uint32_t r = blockIdx.x;
  if (r >= nq) return;
  const int tid = threadIdx.x;
  const SweepIn q = qs[r];
  __shared__ float s_t[QT];
  __shared__ float4 s_p[QT], s_n[QT];
  __shared__ uint8_t s_hit[QT];
  __shared__ int done, have;
  __shared__ float b_t;
  __shared__ uint32_t b_code;  // id + 1 or 0xFFFFFFFF (terrain)
  __shared__ f3 b_p, b_n;
  __shared__ int b_over;
  if (tid == 0) { done = 0; have = 0; b_t = 0.0f; b_code = 0; b_over = 0; }
  __syncthreads();
  Shape cap;
  cap.kind = SH_CAPSULE; cap.a = q.r; cap.b = q.hh; cap.c = 0.0f;
  Iso cx;
  cx.pos = q.from; cx.rot = mkq(0, 0, 0, 1);
  // 1. overlap at t = 0 (queries.rs:133-152): the first collider in order that touches
  for (uint32_t base = 0; base < ncol && !done; base += QT) {
    const uint32_t ci = base + tid;
    bool hit = false;
    if (ci < ncol) {
      const uint32_t bd = cbody[ci];
      if (alive[bd] && bd != q.ignore) {
        const float4 d = cdims[ci];
        Shape sh; sh.kind = ckind[ci]; sh.a = d.x; sh.b = d.y; sh.c = d.z;
        Iso bx; bx.pos = xyz(pos[bd]); bx.rot = asq(rot[bd]);
        Manifold m;
        if (collide_pair(cap, cx, sh, bx, 0.0f, &m) && m.len > 0) {
          hit = true;
          s_p[tid] = f4(m.pts[0].position);
          s_n[tid] = f4(m.normal);
        }
      }
    }
    s_hit[tid] = hit ? 1 : 0;
    __syncthreads();
    if (tid == 0) {
      for (int k = 0; k < QT; ++k)
        if (s_hit[k]) {
          done = 1; have = 1; b_over = 1; b_t = 0.0f; b_code = cbody[base + k] + 1u;
          b_p = xyz(s_p[k]); b_n = xyz(s_n[k]);
          break;
        }
    }
    __syncthreads();
  }
  // terrain triangles at t = 0 (queries.rs:154-175): the capsule's AABB window, first overlap
  auto window = [&](f3 qmn, f3 qmx, long long* gx0, long long* gx1, long long* gz0, long long* gz1) {
    return hf_window(hf, qmn, qmx, gx0, gx1, gz0, gz1);
  };
  auto tri_of = [&](long long gx0, unsigned long long wx, long long gz0, unsigned long long k, Tri* t) {
    hf_tri(hf, gx0, wx, gz0, k, t);
  };
  if (has_hf && !done) {
    f3 mn, mx;
    aabb_of(SH_CAPSULE, make_float4(q.r, q.hh, 0.0f, 0.0f), q.from, mkq(0, 0, 0, 1), &mn, &mx);
    long long gx0, gx1, gz0, gz1;
    if (window(mn, mx, &gx0, &gx1, &gz0, &gz1)) {
      const unsigned long long wx = (unsigned long long)(gx1 - gx0 + 1), ntri = 2ull * wx * (unsigned long long)(gz1 - gz0 + 1);
      for (unsigned long long base = 0; base < ntri && !done; base += QT) {
        const unsigned long long k = base + tid;
        bool hit = false;
        if (k < ntri) {
          Tri t;
          tri_of(gx0, wx, gz0, k, &t);
          Manifold m;
          if (collide_tri(cap, cx, t, 0.0f, &m) && m.len > 0) { hit = true; s_p[tid] = f4(m.pts[0].position); s_n[tid] = f4(m.normal); }
        }
        s_hit[tid] = hit ? 1 : 0;
        __syncthreads();
        if (tid == 0) {
          for (int k2 = 0; k2 < QT; ++k2)
            if (s_hit[k2]) {
              done = 1; have = 1; b_over = 1; b_t = 0.0f; b_code = 0xFFFFFFFFu;
              b_p = xyz(s_p[k2]); b_n = xyz(s_n[k2]);
              break;
            }
        }
        __syncthreads();
      }
    }
  }
  const f3 v = q.to - q.from;
  if (!done && !(len2(v) < 1.0e-12f)) {
    // 2. the swept tip and base spheres against the colliders' AABBs (queries.rs:179-212)
    const f3 tip0 = q.from + mk3(0.0f, q.hh, 0.0f), base0 = q.from + mk3(0.0f, -q.hh, 0.0f);
    __shared__ uint32_t b_ci;
    __shared__ int s_kind[QT];
    if (tid == 0) b_ci = 0;
    for (uint32_t base = 0; base < ncol; base += QT) {
      const uint32_t ci = base + tid;
      bool hit = false;
      if (ci < ncol) {
        const uint32_t bd = cbody[ci];
        if (alive[bd] && bd != q.ignore) {
          f3 mn, mx;
          aabb_of(ckind[ci], cdims[ci], xyz(pos[bd]), asq(rot[bd]), &mn, &mx);
          float t;
          f3 n;
          int kind;
          if (sweep_two(tip0, base0, v, q.r, mn, mx, &t, &n, &kind)) {
            t = clampf(t, 0.0f, 1.0f);
            const f3 c0 = kind == 0 ? tip0 : base0;
            hit = true;
            s_t[tid] = t; s_n[tid] = f4(n); s_p[tid] = f4((c0 + v * t) - n * q.r); s_kind[tid] = kind;
          }
        }
      }
      s_hit[tid] = hit ? 1 : 0;
      __syncthreads();
      if (tid == 0) {
        for (int k = 0; k < QT; ++k) {
          if (!s_hit[k]) continue;
          const float t = s_t[k];
          const uint32_t ci2 = base + k;
          if (!have || (t < b_t - kToiEps) || (fabsf(t - b_t) <= kToiEps && ci2 < b_ci)) {
            have = 1; b_t = t; b_ci = ci2; b_code = cbody[ci2] + 1u; b_p = xyz(s_p[k]); b_n = xyz(s_n[k]);
          }
        }
      }
      __syncthreads();
    }
    // the terrain triangles' AABBs in the swept box (queries.rs:214-236)
    if (has_hf) {
      const f3 ext = splat(q.r + q.hh);
      f3 qa = vmin(q.from, q.to) - ext, qb = vmax(q.from, q.to) + ext;
      qa = mk3(qf32(qa.x), qf32(qa.y), qf32(qa.z));
      qb = mk3(qf32(qb.x), qf32(qb.y), qf32(qb.z));
      long long gx0, gx1, gz0, gz1;
      if (window(vmin(qa, qb), vmax(qa, qb), &gx0, &gx1, &gz0, &gz1)) {
        const unsigned long long wx = (unsigned long long)(gx1 - gx0 + 1), ntri = 2ull * wx * (unsigned long long)(gz1 - gz0 + 1);
        for (unsigned long long base = 0; base < ntri; base += QT) {
          const unsigned long long k = base + tid;
          bool hit = false;
          if (k < ntri) {
            Tri tr;
            tri_of(gx0, wx, gz0, k, &tr);
            // aabb_of(Triangle, identity) (shape.rs:60-70): the vertices through the identity pose
            const q4 id = mkq(0, 0, 0, 1);
            const f3 wa = mk3(0, 0, 0) + qrot(id, tr.a), wb = mk3(0, 0, 0) + qrot(id, tr.b), wc = mk3(0, 0, 0) + qrot(id, tr.c);
            f3 a = vmin(vmin(wa, wb), wc), b = vmax(vmax(wa, wb), wc);
            a = mk3(qf32(a.x), qf32(a.y), qf32(a.z));
            b = mk3(qf32(b.x), qf32(b.y), qf32(b.z));
            const f3 mn = vmin(a, b), mx = vmax(a, b);
            float t;
            f3 n;
            int kind;
            if (sweep_two(tip0, base0, v, q.r, mn, mx, &t, &n, &kind)) {
              t = clampf(t, 0.0f, 1.0f);
              const f3 c0 = kind == 0 ? tip0 : base0;
              hit = true;
              s_t[tid] = t; s_n[tid] = f4(n); s_p[tid] = f4((c0 + v * t) - n * q.r);
            }
          }
          s_hit[tid] = hit ? 1 : 0;
          __syncthreads();
          if (tid == 0) {
            for (int k2 = 0; k2 < QT; ++k2) {
              if (!s_hit[k2]) continue;
              const float t = s_t[k2];
              if (!have || t < b_t - kToiEps) { have = 1; b_t = t; b_code = 0xFFFFFFFFu; b_p = xyz(s_p[k2]); b_n = xyz(s_n[k2]); }
            }
          }
          __syncthreads();
        }
      }
    }
  }
  if (tid == 0) {
    if (!have) {
      out_pt[r] = make_float4(0, 0, 0, __uint_as_float(0u));
      out_n[r] = make_float4(0, 1, 0, 1.0f);
    } else {
      out_pt[r] = make_float4(b_p.x, b_p.y, b_p.z, __uint_as_float(b_code));
      out_n[r] = make_float4(b_n.x, b_n.y, b_n.z, b_over ? -0.0f : clampf(b_t, 0.0f, 1.0f));
    }
  }
}


// ---- exact ray casts: ray_shape (riftphys-geom/src/raycast.rs:13-130), in the shape's frame
__device__ bool ray_sphere_local(f3 o, f3 d, f3 c, float r, float* t_out, f3* n_out) {  // raycast.rs:42-53
  const f3 m = o - c;
  const float b = dot(m, d);
  const float cc = dot(m, m) - r * r;
  if (cc <= 0.0f) { *t_out = 0.0f; *n_out = mk3(-d.x, -d.y, -d.z); return true; }
  if (b > 0.0f) return false;
  const float disc = b * b - cc;
  if (disc < 0.0f) return false;
  const float t = rmax(-b - sqrtf(disc), 0.0f);
  *t_out = t;
  *n_out = normalize_or_zero(m + d * t);
  return true;
}
__device__ bool ray_box_local(f3 o, f3 d, f3 he, float* t_out, f3* n_out) {  // raycast.rs:55-82
  float tmin = 0.0f, tmax = __int_as_float(0x7f800000);
  f3 normal = mk3(-d.x, -d.y, -d.z);
  const float oa[3] = {o.x, o.y, o.z}, da[3] = {d.x, d.y, d.z}, ha[3] = {he.x, he.y, he.z};
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    if (fabsf(da[ax]) < 1.0e-9f) {
      if (oa[ax] < -ha[ax] || oa[ax] > ha[ax]) return false;
      continue;
    }
    const float inv = 1.0f / da[ax];
    float t1 = (-ha[ax] - oa[ax]) * inv, t2 = (ha[ax] - oa[ax]) * inv;
    float sign = -1.0f;
    if (t1 > t2) { const float sw = t1; t1 = t2; t2 = sw; sign = 1.0f; }
    if (t1 > tmin) {
      tmin = t1;
      normal = mk3(ax == 0 ? sign : 0.0f, ax == 1 ? sign : 0.0f, ax == 2 ? sign : 0.0f);
    }
    tmax = rmin(tmax, t2);
    if (tmin > tmax) return false;
  }
  *t_out = tmin;
  *n_out = normal;
  return true;
}
__device__ bool ray_tube_local(f3 o, f3 d, float r, float hh, float* t_out, f3* n_out) {  // raycast.rs:84-96
  const float a = d.x * d.x + d.z * d.z;
  if (a < 1.0e-9f) return false;
  const float b = o.x * d.x + o.z * d.z;
  const float c = o.x * o.x + o.z * o.z - r * r;
  const float disc = b * b - a * c;
  if (disc < 0.0f) return false;
  const float t = (-b - sqrtf(disc)) / a;
  if (t < 0.0f) return false;
  const f3 p = o + d * t;
  if (fabsf(p.y) > hh) return false;
  *t_out = t;
  *n_out = normalize_or_zero(mk3(p.x, 0.0f, p.z));
  return true;
}
__device__ bool ray_capsule_local(f3 o, f3 d, float r, float hh, float* t_out, f3* n_out) {  // raycast.rs:98-109
  const f3 oc = o - mk3(0.0f, clampf(o.y, -hh, hh), 0.0f);
  if (dot(oc, oc) <= r * r) { *t_out = 0.0f; *n_out = mk3(-d.x, -d.y, -d.z); return true; }
  bool have = ray_tube_local(o, d, r, hh, t_out, n_out);
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    float t;
    f3 n;
    if (ray_sphere_local(o, d, mk3(0.0f, e == 0 ? hh : -hh, 0.0f), r, &t, &n) && (!have || t < *t_out)) {
      have = true; *t_out = t; *n_out = n;
    }
  }
  return have;
}
// ray_shape: kind 0 sphere, 1 box, 2 capsule (dims as the colliders'), 3 the triangle tri
__device__ bool ray_shape_dev(uint32_t kind, float4 dims, const Tri& tri, f3 xp, q4 xq, f3 origin, f3 dir, float max_t,
                              float* t_out, f3* n_out) {
  if (!(max_t >= 0.0f) || !vfin(origin) || !vfin(dir)) return false;
  const q4 inv = qconj(xq);
  const f3 o = qrot(inv, origin - xp), d = qrot(inv, dir);
  float t = 0.0f;
  f3 n = mk3(0, 0, 0);
  bool hit;
  if (kind == SH_SPHERE) hit = ray_sphere_local(o, d, mk3(0, 0, 0), fabsf(dims.x), &t, &n);
  else if (kind == SH_BOX) hit = ray_box_local(o, d, mk3(fabsf(dims.x), fabsf(dims.y), fabsf(dims.z)), &t, &n);
  else if (kind == SH_CAPSULE) hit = ray_capsule_local(o, d, fabsf(dims.x), fabsf(dims.y), &t, &n);
  else {
    hit = ray_triangle(o, d, max_t, tri.a, tri.b, tri.c, &t);
    if (hit) {
      const f3 tn = tri_normal(tri.a, tri.b, tri.c);
      n = dot(tn, d) > 0.0f ? mk3(-tn.x, -tn.y, -tn.z) : tn;
    }
  }
  if (!hit || !(t <= max_t && fin(t))) return false;
  *t_out = t;
  *n_out = qrot(xq, n);
  return true;
}

// World::raycast_exact (queries.rs:18-48): colliders whose fresh AABB the ray meets, tested against
// their true shape, then the heightfield's triangles in the ray's box; a hit replaces the best only
// when strictly nearer, so the first of equals (lowest collider, colliders before terrain) stays.
__global__ void __launch_bounds__(QT) k_raycast_exact(uint32_t nrays, const RayIn* __restrict__ rays, uint32_t ncol,
                                                      const uint32_t* __restrict__ cbody, const uint32_t* __restrict__ ckind,
                                                      const float4* __restrict__ cdims, const float4* __restrict__ pos,
                                                      const float4* __restrict__ rot, const uint8_t* __restrict__ alive,
                                                      bool has_hf, HfDev hf, float4* out_pt, float4* out_n) {
  const uint32_t r = blockIdx.x;
  if (r >= nrays) return;
  const int tid = threadIdx.x;
  const RayIn ray = rays[r];
  __shared__ float s_t[QT];
  __shared__ float4 s_n[QT];
  __shared__ uint8_t s_hit[QT];
  __shared__ float b_t;
  __shared__ uint32_t b_code;
  __shared__ f3 b_n;
  __shared__ int have;
  if (tid == 0) { have = 0; b_t = 0.0f; b_code = 0; }
  __syncthreads();
  const Tri none{};
  for (uint32_t base = 0; base < ncol; base += QT) {
    const uint32_t ci = base + tid;
    bool hit = false;
    if (ci < ncol) {
      const uint32_t bd = cbody[ci];
      if (alive[bd] && bd != ray.ignore) {
        const f3 bp = xyz(pos[bd]);
        const q4 bq = asq(rot[bd]);
        f3 mn, mx, p0, n0;
        float t0;
        aabb_of(ckind[ci], cdims[ci], bp, bq, &mn, &mx);
        if (ray_aabb(ray.o, ray.d, mn, mx, ray.max_d, &t0, &p0, &n0)) {
          float t;
          f3 n;
          hit = ray_shape_dev(ckind[ci], cdims[ci], none, bp, bq, ray.o, ray.d, ray.max_d, &t, &n);
          if (hit) { s_t[tid] = t; s_n[tid] = f4(n); }
        }
      }
    }
    s_hit[tid] = hit ? 1 : 0;
    __syncthreads();
    if (tid == 0) {
      for (int k = 0; k < QT; ++k) {
        if (!s_hit[k] || (have && !(s_t[k] < b_t))) continue;
        have = 1; b_t = s_t[k]; b_code = cbody[base + k] + 1u; b_n = xyz(s_n[k]);
      }
    }
    __syncthreads();
  }
  if (has_hf) {
    const f3 end = ray.o + ray.d * ray.max_d;
    f3 qa = vmin(ray.o, end), qb = vmax(ray.o, end);
    qa = mk3(qf32(qa.x), qf32(qa.y), qf32(qa.z));
    qb = mk3(qf32(qb.x), qf32(qb.y), qf32(qb.z));
    long long gx0, gx1, gz0, gz1;
    if (hf_window(hf, vmin(qa, qb), vmax(qa, qb), &gx0, &gx1, &gz0, &gz1)) {
      const unsigned long long wx = (unsigned long long)(gx1 - gx0 + 1), ntri = 2ull * wx * (unsigned long long)(gz1 - gz0 + 1);
      const q4 qid = mkq(0, 0, 0, 1);
      for (unsigned long long base = 0; base < ntri; base += QT) {
        const unsigned long long k = base + tid;
        bool hit = false;
        if (k < ntri) {
          Tri tr;
          hf_tri(hf, gx0, wx, gz0, k, &tr);
          float t;
          f3 n;
          hit = ray_shape_dev(3u, make_float4(0, 0, 0, 0), tr, mk3(0, 0, 0), qid, ray.o, ray.d, ray.max_d, &t, &n);
          if (hit) { s_t[tid] = t; s_n[tid] = f4(n); }
        }
        s_hit[tid] = hit ? 1 : 0;
        __syncthreads();
        if (tid == 0) {
          for (int q = 0; q < QT; ++q) {
            if (!s_hit[q] || (have && !(s_t[q] < b_t))) continue;
            have = 1; b_t = s_t[q]; b_code = 0xFFFFFFFFu; b_n = xyz(s_n[q]);
          }
        }
        __syncthreads();
      }
    }
  }
  if (tid == 0) {
    if (!have) {
      out_pt[r] = make_float4(0, 0, 0, __uint_as_float(0u));
      out_n[r] = make_float4(0, 1, 0, 1.0f);
    } else {
      const f3 p = ray.o + ray.d * b_t;
      out_pt[r] = make_float4(p.x, p.y, p.z, __uint_as_float(b_code));
      out_n[r] = make_float4(b_n.x, b_n.y, b_n.z, clampf(b_t / ray.max_d, 0.0f, 1.0f));
    }
  }
}

// World::sweep_capsule over a batch: per query from xyz, to xyz, radius, half height, ignored body
// index bits (0xFFFFFFFF: none) and 3 words of padding; out as raycast_batch's, with the normal's
// w = -0.0 when the capsule started overlapping (toi 0).
void WorldGpu::sweep_batch(uint32_t n, const float* q12, float4* hit_pt, float4* hit_n) {
  auto& S = *s_;
  cudaStream_t st = stream_;
  if (n == 0) return;
  S.ray_in.ensure(3ull * n + 3);
  S.ray_pt.ensure(n + 1);
  S.ray_n.ensure(n + 1);
  RP_CUDA(cudaMemcpyAsync(S.ray_in.p, q12, sizeof(SweepIn) * n, cudaMemcpyHostToDevice, st));
  HfDev hf{hf_h_.p, hf_nx_, hf_nz_, hf_sx_, hf_sz_, hf_ox_, hf_oz_, hf_min_, hf_max_};
  k_sweep<<<n, QT, 0, st>>>(n, reinterpret_cast<const SweepIn*>(S.ray_in.p), ncol_, col_body.p, col_kind.p, col_dims.p,
                             pos.p, rot.p, alive_d.p, has_hf_, hf, S.ray_pt.p, S.ray_n.p);
  RP_COUNT_LAUNCH(1);
  RP_CUDA(cudaMemcpyAsync(hit_pt, S.ray_pt.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaMemcpyAsync(hit_n, S.ray_n.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
}

// World::raycast over a batch (queries.rs:50-116): n rays with origin, direction (unit) and max
// distance; out per ray (x y z, body id + 1 bits or 0 for none or 0xFFFFFFFF for the terrain)
// and (normal, fraction).
void WorldGpu::raycast_batch(uint32_t n, const float* rays8, float4* hit_pt, float4* hit_n, bool exact) {
  auto& S = *s_;
  cudaStream_t st = stream_;
  if (n == 0) return;
  S.ray_in.ensure(2ull * n + 2);
  S.ray_pt.ensure(n + 1);
  S.ray_n.ensure(n + 1);
  RP_CUDA(cudaMemcpyAsync(S.ray_in.p, rays8, sizeof(RayIn) * n, cudaMemcpyHostToDevice, st));
  HfDev hf{hf_h_.p, hf_nx_, hf_nz_, hf_sx_, hf_sz_, hf_ox_, hf_oz_, hf_min_, hf_max_};
  if (exact)
    k_raycast_exact<<<n, QT, 0, st>>>(n, reinterpret_cast<const RayIn*>(S.ray_in.p), ncol_, col_body.p, col_kind.p,
                                       col_dims.p, pos.p, rot.p, alive_d.p, has_hf_, hf, S.ray_pt.p, S.ray_n.p);
  else
    k_raycast<<<n, QT, 0, st>>>(n, reinterpret_cast<const RayIn*>(S.ray_in.p), ncol_, col_body.p, col_kind.p, col_dims.p,
                                 pos.p, rot.p, alive_d.p, has_hf_, hf, S.ray_pt.p, S.ray_n.p);
  RP_COUNT_LAUNCH(1);
  RP_CUDA(cudaMemcpyAsync(hit_pt, S.ray_pt.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaMemcpyAsync(hit_n, S.ray_n.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
}

}  // namespace rp
