// step_front.cu -- stages 1 and 2 of the tick on the GPU: forces, AABBs and swept AABBs,
// the uniform-grid broadphase, pair and terrain narrowphase, contact culling and orientation.
// Reference: riftphys-world/src/world/step.rs:53-150, 499-542; broadphase.rs:29-99;
// narrowphase.rs; terrain.rs:300-358.
#include <cub/cub.cuh>

#include "rp_narrow.cuh"
#include "shape_aabb.cuh"
#include "step_internal.cuh"

namespace rp {

// ------------------------------------------------------------------ stage 1
// Stage 1 forces (step.rs:55-68): snapshot the start-of-step velocities; v += q6(g) dt for
// dynamic awake bodies (grav_eval Uniform, gravity.rs:79-87). One thread per body.
__global__ void k_forces(int nb, const float4* lin, const float4* __restrict__ ang,
                         float4* lin_out, float4* pre_lin, float4* pre_ang,
                         const uint8_t* __restrict__ dyn, const uint8_t* __restrict__ awake, f3 g, float dt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  float4 l = lin[i];
  pre_lin[i] = l;
  pre_ang[i] = ang[i];
  if (!dyn[i] || !awake[i]) return;
  f3 nl = xyz(l) + g * dt;
  if (vfin(nl)) lin_out[i] = f4(fin_v(nl), l.w);  // Bodies::set_vel (dynamics.rs:141-145)
}

// update_colliders_aabb (world.rs:793-798) + the swept, margin-inflated box (step.rs:75-81):
// s = 0.05 + (|v| + |w| reach) dt, reach = half the AABB diagonal (world.rs:97-100).
// Also classifies each collider for the broadphase (broadphase.rs:36-47): 0 = skipped
// (non-finite min.x), 1 = in the grid, 2 = oversized (> 5 cells on an axis).
__global__ void k_aabbs(int ncol, const uint32_t* __restrict__ cbody, const uint32_t* __restrict__ ckind,
                        const float4* __restrict__ cdims, const float4* __restrict__ pos, const float4* __restrict__ rot,
                        const float4* __restrict__ lin, const float4* __restrict__ ang, float dt,
                        float4* amin, float4* amax, float4* smin, float4* smax, float* sweep,
                        uint32_t* sap_flag, uint32_t* over_flag, uint32_t* err) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  uint32_t b = cbody[c];
  f3 mn, mx;
  aabb_of(ckind[c], cdims[c], xyz(pos[b]), asq(rot[b]), &mn, &mx);
  amin[c] = f4(mn);
  amax[c] = f4(mx);
  float reach = 0.5f * len(mx - mn);
  float s = 0.05f + (len(xyz(lin[b])) + len(xyz(ang[b])) * reach) * dt;
  sweep[c] = s;
  f3 a = mn - splat(s), z = mx + splat(s);
  smin[c] = f4(a);
  smax[c] = f4(z);
  uint32_t cls = 0;
  if (fin(a.x)) {
    float dx = z.x - a.x, dy = z.y - a.y, dz = z.z - a.z;
    const float lim = 2.5f * 5.0f;
    if (dx > lim || dy > lim || dz > lim) cls = 2;
    else {
      cls = 1;
      if (!(fin(a.y) && fin(a.z) && fin(z.x) && fin(z.y) && fin(z.z))) atomicOr(err, 1u);
    }
  }
  sap_flag[c] = cls == 1;
  over_flag[c] = cls == 2;
}

// ------------------------------------------------------------------ broadphase
__device__ __forceinline__ bool overlaps4(float4 amn, float4 amx, float4 bmn, float4 bmx) {
  return !(amx.x < bmn.x || amn.x > bmx.x || amx.y < bmn.y || amn.y > bmx.y || amx.z < bmn.z || amn.z > bmx.z);
}
// ------------------------------------------------------------------ uniform grid (2.5 m cells)
// The reference's own grid (broadphase.rs:29-81): each in-grid collider goes into every cell its
// swept AABB spans (cell = floor(v / 2.5) as i32, saturating, NaN -> 0); colliders sharing a cell
// are tested with the inclusive overlap. On the GPU the (world, cell) keys are sorted, and a
// pair is emitted only from its home cell -- the cell of the min corner of the two AABBs'
// intersection, which both span -- so each overlapping pair comes out once per home-cell key
// (a later sort + unique removes any repeats). Cell coordinates are packed 14 bits each
// (wrapping beyond +-8192 cells only merges distant cells into one key: more tests, same set).
#define GRID_CELL 2.5f
__device__ __forceinline__ int grid_cell(float v) {
  float f = floorf(v / GRID_CELL);
  if (isnan(f)) return 0;
  if (f >= 2147483647.0f) return 2147483647;
  if (f <= -2147483648.0f) return (int)0x80000000;
  return (int)f;
}
__device__ __forceinline__ unsigned long long grid_key(uint32_t world, int x, int y, int z) {
  return ((unsigned long long)world << 42) | ((unsigned long long)((uint32_t)(x + 8192) & 0x3FFFu) << 28) |
         ((unsigned long long)((uint32_t)(y + 8192) & 0x3FFFu) << 14) | (unsigned long long)((uint32_t)(z + 8192) & 0x3FFFu);
}
// cell range of one dimension, at most 6 cells (an in-grid AABB spans <= 12.5 m; more means a
// non-finite extent, already flagged by k_aabbs)
__device__ __forceinline__ void grid_span(float lo, float hi, int* c0, int* n) {
  int a = grid_cell(lo), b = grid_cell(hi);
  long long w = (long long)b - (long long)a + 1;
  *c0 = a;
  *n = w < 0 ? 0 : (w > 6 ? 6 : (int)w);
}
__global__ void k_grid_count(int n, const uint32_t* __restrict__ ids, const float4* __restrict__ smin,
                             const float4* __restrict__ smax, uint32_t* cnt) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t c = ids[k];
  float4 mn = smin[c], mx = smax[c];
  int x0, nx, y0, ny, z0, nz;
  grid_span(mn.x, mx.x, &x0, &nx); grid_span(mn.y, mx.y, &y0, &ny); grid_span(mn.z, mx.z, &z0, &nz);
  cnt[k] = (uint32_t)(nx * ny * nz);
}
__global__ void k_grid_emit(int n, const uint32_t* __restrict__ ids, const float4* __restrict__ smin,
                            const float4* __restrict__ smax, const uint32_t* __restrict__ col_world,
                            const uint32_t* __restrict__ off, unsigned long long* keys, uint32_t* vals) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t c = ids[k], w = col_world ? col_world[c] : 0u;
  float4 mn = smin[c], mx = smax[c];
  int x0, nx, y0, ny, z0, nz;
  grid_span(mn.x, mx.x, &x0, &nx); grid_span(mn.y, mx.y, &y0, &ny); grid_span(mn.z, mx.z, &z0, &nz);
  uint32_t o = off[k];
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        keys[o] = grid_key(w, x0 + x, y0 + y, z0 + z);
        vals[o] = c;
        o++;
      }
}
template <bool EMIT>
__global__ void k_grid_pairs(uint32_t n, const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ vals,
                             const float4* __restrict__ smin, const float4* __restrict__ smax,
                             const uint32_t* __restrict__ col_world, uint32_t* cnt, const uint32_t* __restrict__ off,
                             unsigned long long* out) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const unsigned long long key = keys[e];
  const uint32_t i = vals[e];
  const float4 imn = smin[i], imx = smax[i];
  const uint32_t w = col_world ? col_world[i] : 0u;
  uint32_t c = 0, o = EMIT ? off[e] : 0;
  for (uint32_t f = e + 1; f < n && keys[f] == key; ++f) {
    uint32_t j = vals[f];
    if (j == i) continue;
    float4 jmn = smin[j], jmx = smax[j];
    if (!overlaps4(imn, imx, jmn, jmx)) continue;
    unsigned long long home = grid_key(w, grid_cell(fmaxf(imn.x, jmn.x)), grid_cell(fmaxf(imn.y, jmn.y)),
                                       grid_cell(fmaxf(imn.z, jmn.z)));
    if (home != key) continue;
    if (EMIT) {
      uint32_t lo = i < j ? i : j, hi = i < j ? j : i;
      out[o + c] = ((unsigned long long)lo << 32) | hi;
    }
    c++;
  }
  if (!EMIT) cnt[e] = c;
}

// Oversized colliders against every collider (broadphase.rs:83-92), one thread per collider.
// Batched worlds: only the oversized colliders of c's own world (a contiguous run of the
// collider-ordered list, found by binary search on the world's collider range).
__device__ __forceinline__ int lower_bound_u32(const uint32_t* a, int n, uint32_t v) {
  int lo = 0, hi = n;
  while (lo < hi) { int m = (lo + hi) >> 1; if (a[m] < v) lo = m + 1; else hi = m; }
  return lo;
}
template <bool EMIT>
__global__ void k_oversized(int ncol, int nover, const uint32_t* __restrict__ over, const float4* __restrict__ smin,
                            const float4* __restrict__ smax, uint32_t* cnt, const uint32_t* __restrict__ off,
                            unsigned long long* out, const uint32_t* __restrict__ col_world = nullptr,
                            const uint32_t* __restrict__ world_col_start = nullptr) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  float4 cmn = smin[c], cmx = smax[c];
  uint32_t k = 0, o = EMIT ? off[c] : 0;
  int t0 = 0, t1 = nover;
  if (col_world) {
    uint32_t w = col_world[c];
    t0 = lower_bound_u32(over, nover, world_col_start[w]);
    t1 = lower_bound_u32(over, nover, world_col_start[w + 1]);
  }
  for (int t = t0; t < t1; ++t) {
    uint32_t b = over[t];
    if (b == (uint32_t)c) continue;
    if (overlaps4(smin[b], smax[b], cmn, cmx)) {
      if (EMIT) {
        uint32_t lo = b < (uint32_t)c ? b : c, hi = b < (uint32_t)c ? c : b;
        out[o + k] = ((unsigned long long)lo << 32) | hi;
      }
      k++;
    }
  }
  if (!EMIT) cnt[c] = k;
}
__global__ void k_unique_flags(int n, const unsigned long long* __restrict__ a, uint8_t* flag) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) flag[k] = (k == 0 || a[k] != a[k - 1]) ? 1 : 0;
}

// ------------------------------------------------------------------ narrowphase
// Bodies joined by a joint (step.rs:85-102): binary search of (min << 32 | max) in the sorted keys.
__device__ __forceinline__ bool jointed_pair(uint32_t a, uint32_t b, const unsigned long long* __restrict__ keys,
                                             uint32_t n) {
  unsigned long long k = a < b ? (((unsigned long long)a << 32) | b) : (((unsigned long long)b << 32) | a);
  uint32_t lo = 0, hi = n;
  while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (keys[m] < k) lo = m + 1; else hi = m; }
  return lo < n && keys[lo] == k;
}
// One thread per broadphase pair (step.rs:97-113): contact distance reach = s_i + s_j - 0.05;
// depth = penetration - reach + 0.05. Up to 4 points in fixed slots. Same-body and jointed pairs
// make no contact.
__global__ void k_narrow_pairs(int np, const unsigned long long* __restrict__ pairs, const uint32_t* __restrict__ cbody,
                               const uint32_t* __restrict__ ckind, const float4* __restrict__ cdims,
                               const float4* __restrict__ pos, const float4* __restrict__ rot,
                               const float* __restrict__ sweep, const unsigned long long* __restrict__ jkeys,
                               uint32_t njk, float4* out_pt, float4* out_n, uint32_t* out_cnt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  unsigned long long key = pairs[p];
  uint32_t i = (uint32_t)(key >> 32), j = (uint32_t)key;
  uint32_t ba = cbody[i], bb = cbody[j];
  uint32_t cnt = 0;
  if (ba != bb && !(njk && jointed_pair(ba, bb, jkeys, njk))) {
    float reach = sweep[i] + sweep[j] - 0.05f;
    float4 da = cdims[i], db = cdims[j];
    Shape sa; sa.kind = ckind[i]; sa.a = da.x; sa.b = da.y; sa.c = da.z;
    Shape sb; sb.kind = ckind[j]; sb.a = db.x; sb.b = db.y; sb.c = db.z;
    Iso xa; xa.pos = xyz(pos[ba]); xa.rot = asq(rot[ba]);
    Iso xb; xb.pos = xyz(pos[bb]); xb.rot = asq(rot[bb]);
    Manifold m;
    if (collide_pair(sa, xa, sb, xb, reach, &m)) {
      for (int k = 0; k < m.len; ++k) {
        out_pt[4 * p + k] = f4(m.pts[k].position, (m.pts[k].penetration - reach) + 0.05f);
        out_n[4 * p + k] = f4(m.pts[k].normal);
      }
      cnt = m.len;
    }
  }
  out_cnt[p] = cnt;
}

// HeightField::query_aabb (terrain.rs:300-358): the cell window of an AABB.
__device__ __forceinline__ long sat_i32(float f) {
  if (isnan(f)) return 0;
  if (f >= 2147483647.0f) return 2147483647L;
  if (f <= -2147483648.0f) return -2147483648L;
  return (long)f;
}
__device__ __forceinline__ bool hf_window(const HFView& hf, f3 mn, f3 mx, int* gx0, int* gx1, int* gz0, int* gz1) {
  int nx = (int)hf.nx, nz = (int)hf.nz;
  if (nx < 2 || nz < 2) return false;
  float lminx = mn.x - hf.ox, lmaxx = mx.x - hf.ox, lminz = mn.z - hf.oz, lmaxz = mx.z - hf.oz;
  long a = sat_i32(floorf(lminx / hf.sx)) - 1, b = sat_i32(ceilf(lmaxx / hf.sx)) + 1;
  long c = sat_i32(floorf(lminz / hf.sz)) - 1, d = sat_i32(ceilf(lmaxz / hf.sz)) + 1;
  *gx0 = (int)(a < 0 ? 0 : (a > nx - 2 ? nx - 2 : a));
  *gx1 = (int)(b < 0 ? 0 : (b > nx - 2 ? nx - 2 : b));
  *gz0 = (int)(c < 0 ? 0 : (c > nz - 2 ? nz - 2 : c));
  *gz1 = (int)(d < 0 ? 0 : (d > nz - 2 ? nz - 2 : d));
  if (mn.y > hf.max_y + 1.0f || mx.y < hf.min_y - 1.0f) return false;
  return true;
}
__device__ __forceinline__ Tri hf_tri(const HFView& hf, int gx, int gz, int which) {
  float h00 = hf.h[(size_t)gx + (size_t)gz * hf.nx], h10 = hf.h[(size_t)(gx + 1) + (size_t)gz * hf.nx];
  float h01 = hf.h[(size_t)gx + (size_t)(gz + 1) * hf.nx], h11 = hf.h[(size_t)(gx + 1) + (size_t)(gz + 1) * hf.nx];
  float x0 = (float)gx * hf.sx + hf.ox, x1 = x0 + hf.sx;
  float z0 = (float)gz * hf.sz + hf.oz, z1 = z0 + hf.sz;
  Tri t;
  if (which == 0) { t.a = mk3(x0, h00, z0); t.b = mk3(x0, h01, z1); t.c = mk3(x1, h10, z0); }
  else { t.a = mk3(x1, h10, z0); t.b = mk3(x0, h01, z1); t.c = mk3(x1, h11, z1); }
  return t;
}

// Terrain contacts (step.rs:121-141) in three steps, so the triangle narrowphase runs one work
// item per (collider, heightfield cell) instead of one thread per collider:
//   k_terrain_windows  each collider's cell window (HeightField::query_aabb) and its cell count;
//   k_terrain_items    per cell: both triangles through collide_shapes, count (EMIT=false) or
//                      write (EMIT=true) the raw points in query order (gz outer, gx inner,
//                      triangle 1 then 2, manifold order);
//   k_terrain_cull     per collider: cull_and_orient_contacts' bucket rule (step.rs:508-530): up to 4
//                      raw points kept as they are; more: boxes keep reduce_to_4 on the deepest
//                      point's normal, spheres and capsules the 4 deepest by 1e-6 key, earlier first.
__global__ void k_terrain_windows(int ncol, HFView hf, const float4* __restrict__ amin, const float4* __restrict__ amax,
                                  int4* win, uint32_t* ncell) {
  int ci = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= ncol) return;
  int gx0, gx1, gz0, gz1;
  if (!hf_window(hf, xyz(amin[ci]), xyz(amax[ci]), &gx0, &gx1, &gz0, &gz1)) { ncell[ci] = 0; win[ci] = make_int4(0, 0, 0, 0); return; }
  int wx = gx1 - gx0 + 1, wz = gz1 - gz0 + 1;
  if (wx <= 0 || wz <= 0) { ncell[ci] = 0; win[ci] = make_int4(0, 0, 0, 0); return; }
  win[ci] = make_int4(gx0, gz0, wx, wz);
  ncell[ci] = (uint32_t)wx * (uint32_t)wz;
}
__device__ __forceinline__ uint32_t upper_bound_u32(const uint32_t* a, uint32_t n, uint32_t v) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) { uint32_t mid = (lo + hi) >> 1; if (a[mid] <= v) lo = mid + 1; else hi = mid; }
  return lo;
}
// Each item's points go to its 8 fixed slots (2 triangles x at most 4 points), its count to cnt;
// k_terrain_gather then packs them in item order, so the triangle tests run once.
__global__ void k_terrain_items(uint32_t nitems, int ncol, HFView hf, const uint32_t* __restrict__ cell_off,
                                const int4* __restrict__ win, const uint32_t* __restrict__ cbody,
                                const uint32_t* __restrict__ ckind, const float4* __restrict__ cdims,
                                const float4* __restrict__ pos, const float4* __restrict__ rot,
                                const float* __restrict__ sweep, uint32_t* cnt, float4* slot_p, float4* slot_n) {
  uint32_t it = blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= nitems) return;
  uint32_t ci = upper_bound_u32(cell_off, (uint32_t)ncol, it) - 1;  // cell_off: exclusive scan of cell counts
  uint32_t q = it - cell_off[ci];
  int4 w = win[ci];
  int gx = w.x + (int)(q % (uint32_t)w.z);
  int gz = w.y + (int)(q / (uint32_t)w.z);
  uint32_t b = cbody[ci];
  float4 d = cdims[ci];
  Shape sh; sh.kind = ckind[ci]; sh.a = d.x; sh.b = d.y; sh.c = d.z;
  Iso x; x.pos = xyz(pos[b]); x.rot = asq(rot[b]);
  float cd = sweep[ci];
  uint32_t n = 0;
  const size_t o = 8 * (size_t)it;
  for (int tri = 0; tri < 2; ++tri) {
    Tri t = hf_tri(hf, gx, gz, tri);
    Manifold m;
    if (!collide_tri(sh, x, t, cd, &m)) continue;
    for (int k = 0; k < m.len; ++k) {
      slot_p[o + n] = f4(m.pts[k].position, (m.pts[k].penetration - cd) + 0.05f);
      slot_n[o + n] = f4(m.pts[k].normal);
      n++;
    }
  }
  cnt[it] = n;
}
__global__ void k_terrain_gather(uint32_t nitems, const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ cand_off,
                                 const float4* __restrict__ slot_p, const float4* __restrict__ slot_n, float4* cand_p,
                                 float4* cand_n) {
  uint32_t it = blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= nitems) return;
  const uint32_t n = cnt[it], o = cand_off[it];
  for (uint32_t k = 0; k < n; ++k) {
    cand_p[o + k] = slot_p[8 * (size_t)it + k];
    cand_n[o + k] = slot_n[8 * (size_t)it + k];
  }
}
__global__ void k_terrain_cull(int ncol, const uint32_t* __restrict__ ckind, const uint32_t* __restrict__ cell_off,
                               const uint32_t* __restrict__ ncell, const uint32_t* __restrict__ cand_off, uint32_t nitems,
                               uint32_t ncand, const float4* __restrict__ cand_p, const float4* __restrict__ cand_n,
                               float4* out_pt, float4* out_n, uint32_t* out_cnt) {
  int ci = blockIdx.x * blockDim.x + threadIdx.x;
  if (ci >= ncol) return;
  uint32_t i0 = cell_off[ci], i1 = i0 + ncell[ci];
  uint32_t c0 = i0 < nitems ? cand_off[i0] : ncand, c1 = i1 < nitems ? cand_off[i1] : ncand;
  uint32_t total = c1 - c0;
  if (total <= 4) {
    for (uint32_t k = 0; k < total; ++k) { out_pt[4 * ci + k] = cand_p[c0 + k]; out_n[4 * ci + k] = cand_n[c0 + k]; }
    out_cnt[ci] = total;
    return;
  }
  if (ckind[ci] != SH_BOX) {
    // the 4 deepest by 1e-6 key, earlier first on ties (a stable sort by Reverse(key), truncated)
    long long tk[4]; uint32_t ti[4]; int nt = 0;
    for (uint32_t c = c0; c < c1; ++c) {
      long long key = sort_key6(cand_p[c].w);
      int at = nt;
      while (at > 0 && tk[at - 1] < key) at--;
      if (at < 4) {
        int last = nt < 4 ? nt : 3;
        for (int j = last; j > at; --j) { tk[j] = tk[j - 1]; ti[j] = ti[j - 1]; }
        tk[at] = key; ti[at] = c;
        if (nt < 4) nt++;
      }
    }
    for (int k = 0; k < 4; ++k) { out_pt[4 * ci + k] = cand_p[ti[k]]; out_n[4 * ci + k] = cand_n[ti[k]]; }
    out_cnt[ci] = 4;
    return;
  }
  // boxes: reduce_to_4 (narrowphase.rs:312-338) on the deepest point's normal (lowest index on ties)
  auto argmax = [&](int pass, f3 p0, f3 e, f3 nd, float s2, uint32_t* bi, float* bv) {
    long long bk = LLONG_MIN; *bi = c0; *bv = -INFINITY;
    for (uint32_t c = c0; c < c1; ++c) {
      float4 P = cand_p[c];
      f3 pt = xyz(P);
      float v;
      if (pass == 0) v = P.w;
      else if (pass == 1) v = len2(pt - p0);
      else if (pass == 2) v = fabsf(dot(cross(pt - p0, e), nd));
      else v = -dot(cross(pt - p0, e), nd) * s2;
      long long key = sort_key6(v);
      if (key > bk) { bk = key; *bi = c; *bv = v; }
    }
  };
  uint32_t sel[4]; int ns = 0;
  uint32_t i; float v;
  argmax(0, mk3(0, 0, 0), mk3(0, 0, 0), mk3(0, 0, 0), 0.0f, &i, &v);
  f3 p0 = xyz(cand_p[i]), nd = xyz(cand_n[i]);
  sel[ns++] = i;
  argmax(1, p0, mk3(0, 0, 0), nd, 0.0f, &i, &v);
  if (v > 1.0e-12f) {
    sel[ns++] = i;
    f3 e = xyz(cand_p[i]) - p0;
    argmax(2, p0, e, nd, 0.0f, &i, &v);
    if (v > 1.0e-12f) {
      sel[ns++] = i;
      float s2 = signum(dot(cross(xyz(cand_p[i]) - p0, e), nd));
      argmax(3, p0, e, nd, s2, &i, &v);
      if (v > 1.0e-12f) sel[ns++] = i;
    }
  }
  for (int k = 0; k < ns; ++k) { out_pt[4 * ci + k] = cand_p[sel[k]]; out_n[4 * ci + k] = cand_n[sel[k]]; }
  out_cnt[ci] = ns;
}

// First pair index whose collider i is >= c, for every c in [0, ncol]: pair buckets of
// collider c precede its terrain bucket in the BTreeMap order (step.rs:500-505).
__global__ void k_pair_starts(int ncol, int np, const unsigned long long* __restrict__ pairs, uint32_t* pstart) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ncol) return;
  unsigned long long key = (unsigned long long)c << 32;
  int lo = 0, hi = np;
  while (lo < hi) { int mid = (lo + hi) >> 1; if (pairs[mid] < key) lo = mid + 1; else hi = mid; }
  pstart[c] = lo;
}
// Bucket counts in merged key order: pair p at p + i, terrain bucket of c at c + pstart[c+1].
__global__ void k_bucket_counts(int np, int ncol, const unsigned long long* __restrict__ pairs,
                                const uint32_t* __restrict__ pcnt, const uint32_t* __restrict__ tcnt,
                                const uint32_t* __restrict__ pstart, uint32_t* bcnt) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < np) { uint32_t i = (uint32_t)(pairs[k] >> 32); bcnt[k + i] = pcnt[k]; }
  else if (k < np + ncol) { int c = k - np; bcnt[c + pstart[c + 1]] = tcnt ? tcnt[c] : 0; }
}
// Scatter the culled contacts into solve order and orient pair normals from A's collider
// centre toward B's (step.rs:532-540).
__global__ void k_scatter_contacts(int np, int ncol, const unsigned long long* __restrict__ pairs,
                                   const uint32_t* __restrict__ pcnt, const float4* __restrict__ ppt,
                                   const float4* __restrict__ pn, const uint32_t* __restrict__ tcnt,
                                   const float4* __restrict__ tpt, const float4* __restrict__ tn,
                                   const uint32_t* __restrict__ pstart, const uint32_t* __restrict__ boff,
                                   const uint32_t* __restrict__ cbody, const float4* __restrict__ pos,
                                   uint32_t* c_a, uint32_t* c_b, float4* c_pt, float4* c_n) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < np) {
    uint32_t i = (uint32_t)(pairs[k] >> 32), j = (uint32_t)pairs[k];
    uint32_t o = boff[k + i], n = pcnt[k];
    f3 pa = xyz(pos[cbody[i]]), pb = xyz(pos[cbody[j]]);
    for (uint32_t q = 0; q < n; ++q) {
      float4 nn = pn[4 * k + q];
      f3 nv = xyz(nn);
      if (dot(nv, pb - pa) < 0.0f) nv = -nv;
      c_a[o + q] = i; c_b[o + q] = j;
      c_pt[o + q] = ppt[4 * k + q];
      c_n[o + q] = f4(nv, 0.0f);
    }
  } else if (k < np + ncol) {
    int c = k - np;
    if (!tcnt) return;
    uint32_t o = boff[c + pstart[c + 1]], n = tcnt[c];
    for (uint32_t q = 0; q < n; ++q) {
      c_a[o + q] = c; c_b[o + q] = 0xFFFFFFFFu;
      c_pt[o + q] = tpt[4 * c + q];
      float4 nn = tn[4 * c + q];
      c_n[o + q] = make_float4(nn.x, nn.y, nn.z, 0.0f);
    }
  }
}

// ------------------------------------------------------------------ host driver
void run_front(WorldGpu& W, StepCtx& ctx) {
  auto& S = *W.s_;
  cudaStream_t st = W.stream();
  const int nb = (int)W.num_bodies(), ncol = (int)W.num_colliders();
  const int T = 256;
  auto& P = S.prof;
  // stage 1
  P.begin(PH_FORCES, st);
  if (nb > 0) {
    k_forces<<<(nb + T - 1) / T, T, 0, st>>>(nb, W.lin.p, W.ang.p, W.lin.p, S.pre_lin.p, S.pre_ang.p, W.dyn.p,
                                              W.awake.p, ctx.g, ctx.dt); RP_COUNT_LAUNCH(1);
  }
  P.end(PH_FORCES, st);
  P.begin(PH_AABB, st);
  // stage 2: AABBs, sweep, classification
  S.amin.ensure(ncol); S.amax.ensure(ncol); S.smin.ensure(ncol); S.smax.ensure(ncol); S.sweep.ensure(ncol);
  S.u32a.ensure(ncol + 1); S.u32b.ensure(ncol + 1);
  if (ncol > 0) {
    k_aabbs<<<(ncol + T - 1) / T, T, 0, st>>>(ncol, W.col_body.p, W.col_kind.p, W.col_dims.p, W.pos.p, W.rot.p, W.lin.p,
                                               W.ang.p, ctx.dt, S.amin.p, S.amax.p, S.smin.p, S.smax.p, S.sweep.p,
                                               S.u32a.p, S.u32b.p, W.d_stats.p + STAT_ERR); RP_COUNT_LAUNCH(1);
  }
  P.end(PH_AABB, st);
  P.begin(PH_BROAD, st);
  // broadphase: in-grid colliders sorted along x, oversized list
  S.sap_ids.ensure(ncol + 1); S.over_ids.ensure(ncol + 1); S.counts.ensure(4);
  uint32_t n_sap = 0, n_over = 0;
  if (ncol > 0) {
    select_flagged_iota(S, ncol, S.u32a.p, S.sap_ids.p, S.counts.p + 0, st);
    select_flagged_iota(S, ncol, S.u32b.p, S.over_ids.p, S.counts.p + 1, st);
    uint32_t hc[2];
    cudaMemcpyAsync(hc, S.counts.p, 8, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    n_sap = hc[0]; n_over = hc[1];
  }
  S.sap_cnt.ensure(n_sap + 1); S.sap_off.ensure(n_sap + 1);
  S.ov_cnt.ensure(ncol + 1); S.ov_off.ensure(ncol + 1);
  uint32_t n_sap_pairs = 0, n_ov_pairs = 0, n_ent = 0;
  const bool batched = W.batched();
  const uint32_t* cw = batched ? W.col_world.p : nullptr;
  if (n_sap > 0) {
    // grid entries: one per (collider, spanned cell), sorted by (world, cell) key
    k_grid_count<<<(n_sap + T - 1) / T, T, 0, st>>>(n_sap, S.sap_ids.p, S.smin.p, S.smax.p, S.sap_cnt.p); RP_COUNT_LAUNCH(1);
    n_ent = exclusive_scan_total(S, S.sap_cnt.p, S.sap_off.p, n_sap, st);
    S.sap_key64.ensure(n_ent + 1); S.sap_key64b.ensure(n_ent + 1); S.sap_ord.ensure(n_ent + 1); S.sap_w.ensure(n_ent + 1);
    k_grid_emit<<<(n_sap + T - 1) / T, T, 0, st>>>(n_sap, S.sap_ids.p, S.smin.p, S.smax.p, cw, S.sap_off.p, S.sap_key64.p,
                                                    S.sap_ord.p); RP_COUNT_LAUNCH(1);
    int wbits = 0;
    if (batched) while ((1u << wbits) < W.num_worlds() && wbits < 22) wbits++;
    sort_pairs_u64(S, S.sap_key64.p, S.sap_key64b.p, S.sap_ord.p, S.sap_w.p, n_ent, 0, 42 + wbits, st);
    S.gp_cnt.ensure(n_ent + 1); S.gp_off.ensure(n_ent + 1);
    k_grid_pairs<false><<<(n_ent + T - 1) / T, T, 0, st>>>(n_ent, S.sap_key64b.p, S.sap_w.p, S.smin.p, S.smax.p, cw,
                                                           S.gp_cnt.p, nullptr, nullptr); RP_COUNT_LAUNCH(1);
    n_sap_pairs = exclusive_scan_total(S, S.gp_cnt.p, S.gp_off.p, n_ent, st);
  }
  if (n_over > 0 && ncol > 0) {
    k_oversized<false><<<(ncol + T - 1) / T, T, 0, st>>>(ncol, n_over, S.over_ids.p, S.smin.p, S.smax.p, S.ov_cnt.p,
                                                          nullptr, nullptr, batched ? W.col_world.p : nullptr,
                                                          batched ? W.world_col_start.p : nullptr); RP_COUNT_LAUNCH(1);
    n_ov_pairs = exclusive_scan_total(S, S.ov_cnt.p, S.ov_off.p, ncol, st);
  }
  uint32_t n_raw = n_sap_pairs + n_ov_pairs;
  S.pairs.ensure(n_raw + 1); S.pairs2.ensure(n_raw + 1); S.flag8.ensure(n_raw + 1);
  if (n_sap_pairs > 0) {
    k_grid_pairs<true><<<(n_ent + T - 1) / T, T, 0, st>>>(n_ent, S.sap_key64b.p, S.sap_w.p, S.smin.p, S.smax.p, cw, nullptr,
                                                          S.gp_off.p, S.pairs2.p); RP_COUNT_LAUNCH(1);
  }
  if (n_ov_pairs > 0) {
    k_oversized<true><<<(ncol + T - 1) / T, T, 0, st>>>(ncol, n_over, S.over_ids.p, S.smin.p, S.smax.p, nullptr,
                                                         S.ov_off.p, S.pairs2.p + n_sap_pairs, batched ? W.col_world.p : nullptr,
                                                         batched ? W.world_col_start.p : nullptr); RP_COUNT_LAUNCH(1);
  }
  uint32_t np = 0;
  if (n_raw > 0) {
    sort_keys_u64(S, S.pairs2.p, S.pairs.p, n_raw, st);  // -> S.pairs
    k_unique_flags<<<(n_raw + T - 1) / T, T, 0, st>>>(n_raw, S.pairs.p, S.flag8.p); RP_COUNT_LAUNCH(1);
    np = select_flagged_u64(S, S.pairs.p, S.flag8.p, S.pairs2.p, n_raw, st);
    cudaMemcpyAsync(S.pairs.p, S.pairs2.p, sizeof(unsigned long long) * np, cudaMemcpyDeviceToDevice, st);
  }
  ctx.np = np;
  W.n_pairs = np;
  P.end(PH_BROAD, st);
  P.begin(PH_NARROW, st);
  // narrowphase over pairs
  S.p_pt.ensure(4 * (size_t)np + 4); S.p_n.ensure(4 * (size_t)np + 4); S.p_cnt.ensure(np + 1);
  if (np > 0) {
    k_narrow_pairs<<<(np + 127) / 128, 128, 0, st>>>(np, S.pairs.p, W.col_body.p, W.col_kind.p, W.col_dims.p, W.pos.p,
                                                    W.rot.p, S.sweep.p, W.jpair_keys.p, W.n_jpairs, S.p_pt.p, S.p_n.p,
                                                    S.p_cnt.p); RP_COUNT_LAUNCH(1);
  }
  P.end(PH_NARROW, st);
  P.begin(PH_TERRAIN, st);
  // terrain
  S.t_pt.ensure(4 * (size_t)ncol + 4); S.t_n.ensure(4 * (size_t)ncol + 4); S.t_cnt.ensure(ncol + 1);
  bool terrain = ctx.hf.h != nullptr;
  if (terrain && ncol > 0) {
    S.t_win.ensure(ncol + 1); S.t_ncell.ensure(ncol + 1); S.t_celloff.ensure(ncol + 1);
    k_terrain_windows<<<(ncol + T - 1) / T, T, 0, st>>>(ncol, ctx.hf, S.amin.p, S.amax.p, S.t_win.p, S.t_ncell.p); RP_COUNT_LAUNCH(1);
    uint32_t nitems = exclusive_scan_total(S, S.t_ncell.p, S.t_celloff.p, ncol, st);
    uint32_t ncand = 0;
    S.t_icnt.ensure(nitems + 1); S.t_ioff.ensure(nitems + 1);
    S.t_sp.ensure(8 * (size_t)nitems + 8); S.t_sn.ensure(8 * (size_t)nitems + 8);
    if (nitems > 0) {
      k_terrain_items<<<(nitems + 127) / 128, 128, 0, st>>>(nitems, ncol, ctx.hf, S.t_celloff.p, S.t_win.p, W.col_body.p,
                                                           W.col_kind.p, W.col_dims.p, W.pos.p, W.rot.p, S.sweep.p,
                                                           S.t_icnt.p, S.t_sp.p, S.t_sn.p); RP_COUNT_LAUNCH(1);
      ncand = exclusive_scan_total(S, S.t_icnt.p, S.t_ioff.p, nitems, st);
    }
    S.t_cp.ensure(ncand + 1); S.t_cn.ensure(ncand + 1);
    if (ncand > 0) {
      k_terrain_gather<<<(nitems + 255) / 256, 256, 0, st>>>(nitems, S.t_icnt.p, S.t_ioff.p, S.t_sp.p, S.t_sn.p, S.t_cp.p,
                                                            S.t_cn.p); RP_COUNT_LAUNCH(1);
    }
    k_terrain_cull<<<(ncol + 127) / 128, 128, 0, st>>>(ncol, W.col_kind.p, S.t_celloff.p, S.t_ncell.p, S.t_ioff.p, nitems,
                                                      ncand, S.t_cp.p, S.t_cn.p, S.t_pt.p, S.t_n.p, S.t_cnt.p); RP_COUNT_LAUNCH(1);
  }
  P.end(PH_TERRAIN, st);
  P.begin(PH_CONTACTS, st);
  // merge buckets in key order, scan, scatter
  S.pstart.ensure(ncol + 2);
  k_pair_starts<<<(ncol + 1 + T - 1) / T, T, 0, st>>>(ncol, np, S.pairs.p, S.pstart.p); RP_COUNT_LAUNCH(1);
  uint32_t nbk = np + ncol;
  S.bcnt.ensure(nbk + 1); S.boff.ensure(nbk + 1);
  uint32_t nc = 0;
  if (nbk > 0) {
    k_bucket_counts<<<(nbk + T - 1) / T, T, 0, st>>>(np, ncol, S.pairs.p, S.p_cnt.p, terrain ? S.t_cnt.p : nullptr,
                                                    S.pstart.p, S.bcnt.p); RP_COUNT_LAUNCH(1);
    nc = exclusive_scan_total(S, S.bcnt.p, S.boff.p, nbk, st);
  }
  ctx.nc = nc;
  W.n_contacts = nc;
  S.c_a.ensure(nc + 1); S.c_b.ensure(nc + 1); S.c_pt.ensure(nc + 1); S.c_n.ensure(nc + 1);
  if (nc > 0) {
    k_scatter_contacts<<<(nbk + T - 1) / T, T, 0, st>>>(np, ncol, S.pairs.p, S.p_cnt.p, S.p_pt.p, S.p_n.p,
                                                       terrain ? S.t_cnt.p : nullptr, S.t_pt.p, S.t_n.p, S.pstart.p,
                                                       S.boff.p, W.col_body.p, W.pos.p, S.c_a.p, S.c_b.p, S.c_pt.p,
                                                       S.c_n.p); RP_COUNT_LAUNCH(1);
  }
  P.end(PH_CONTACTS, st);
}

}  // namespace rp
