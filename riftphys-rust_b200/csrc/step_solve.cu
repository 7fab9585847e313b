// step_solve.cu -- stages 3 to 7 of the tick on the GPU.
//
// Exactness argument. The reference solves contacts in level batches (solver.rs:621-642): a row's
// level is one more than the last level of any awake dynamic body it writes, so the rows of one
// level write disjoint bodies and batch order reproduces the serial Gauss-Seidel order bit for
// bit (solver.rs:15-18). Every other order-dependent pass over contacts touches the same bodies
// the same way -- warm-start application (:717-762), the ballistic test (step.rs:180-206), the
// position projection (step.rs:447-497) -- so it runs on the same schedule; the two shock passes
// (solver.rs:964-993, step.rs:450-456) sort rows by height first and get their own schedule.
// Rows split into islands (connected through awake dynamic bodies); one warp owns an island and
// walks its levels with __syncwarp between them, so no two warps ever touch the same body.
#include <atomic>
#include <type_traits>
#include <cub/cub.cuh>

#include "step_internal.cuh"
#include "step_rows.cuh"
#include "joints.cuh"
#include "warm_model.h"

namespace rp {

namespace {
const int T = 256;
// at least one block: every kernel returns early past its n, and a zero grid is a launch error
inline int nblk(uint32_t n, int t = T) { return n ? (int)((n + t - 1) / t) : 1; }
}  // namespace

// ------------------------------------------------------------------ islands (islands.rs:27-93)
__global__ void k_iota(uint32_t n, uint32_t* p) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i;
}
// mode 0: the reference's islands (bodies with inv_mass > 0, asleep or not, islands.rs:266-287);
// mode 1: solve islands (bodies an impulse can move: awake and dynamic; and a sleeping body in a
// joint, which the joint's rows move while the contact reads it).
__global__ void k_union_contacts(uint32_t nc, int mode, const uint32_t* __restrict__ c_a, const uint32_t* __restrict__ c_b,
                                 const uint32_t* __restrict__ cbody, const float* __restrict__ inv_mass,
                                 const uint8_t* __restrict__ awake, const uint8_t* __restrict__ jointed, uint32_t* parent) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc || c_b[k] == 0xFFFFFFFFu) return;
  uint32_t a = cbody[c_a[k]], b = cbody[c_b[k]];
  bool da = inv_mass[a] > 0.0f, db = inv_mass[b] > 0.0f;
  if (mode == 1) {
    // a row with no awake body is not solved: it joins nothing
    if (!((da && awake[a]) || (db && awake[b]))) return;
    da = da && (awake[a] || (jointed && jointed[a]));
    db = db && (awake[b] || (jointed && jointed[b]));
  }
  if (da && db) uf_union(parent, a, b);
}
// route_to_island (islands.rs:316-345): the root each contact lands in, marked.
__global__ void k_ref_island_marks(uint32_t nc, const uint32_t* __restrict__ c_a, const uint32_t* __restrict__ c_b,
                                   const uint32_t* __restrict__ cbody, const float* __restrict__ inv_mass,
                                   uint32_t* parent, uint32_t* mark) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  uint32_t a = cbody[c_a[k]];
  bool da = inv_mass[a] > 0.0f, db = false;
  uint32_t b = 0;
  if (c_b[k] != 0xFFFFFFFFu) { b = cbody[c_b[k]]; db = inv_mass[b] > 0.0f; }
  if (!da && !db) return;
  mark[uf_find(parent, da ? a : b)] = 1;
}

// ------------------------------------------------------------------ rows
// World inverse inertia per body, R I^-1 R^T (dynamics.rs:158-163), once per tick: rotations
// don't change during the velocity solve, so every apply_angular_impulse reads the same matrix.
__global__ void k_world_inertia(uint32_t nb, const float4* __restrict__ rot, const float* __restrict__ inv_mass,
                                const float* __restrict__ inv_I, float* Iw) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  m3 m = inv_mass[i] == 0.0f ? mzero() : world_inertia(asq(rot[i]), ld_m3(inv_I, i));
  st_m3(Iw, i, m);
}

__device__ __forceinline__ float eff_mass(float ia, float ib, const m3& IA, const m3& IB, f3 ra, f3 rb, f3 d) {
  f3 ca = cross(ra, d), cb = cross(rb, d);
  float k = ((ia + ib) + dot(ca, mvec(IA, ca))) + dot(cb, mvec(IB, cb));
  return k > 1.0e-9f ? 1.0f / k : 0.0f;
}
// orthonormal_basis (riftphys-world/src/world/geom.rs:30-38)
__device__ __forceinline__ void orthonormal_basis(f3 n, f3* t1, f3* t2) {
  float ax = fabsf(n.x), ay = fabsf(n.y), az = fabsf(n.z);
  f3 base = (ax <= ay && ax <= az) ? mk3(1, 0, 0) : (ay <= az ? mk3(0, 1, 0) : mk3(0, 0, 1));
  *t1 = normalize_or_zero(cross(base, n));
  *t2 = cross(n, *t1);
}

// Constraint pre-processing (solver.rs:494-590), one thread per contact. Also the anchors in
// body A's frame (solver.rs:728-731) and the island of each row that has a movable body.
__global__ void k_build_rows(uint32_t nc, float dt, const uint32_t* __restrict__ c_a, const uint32_t* __restrict__ c_b,
                             const float4* __restrict__ c_pt, const float4* __restrict__ c_n,
                             const uint32_t* __restrict__ cbody, const uint32_t* __restrict__ cmat, uint32_t hf_mat,
                             const float* __restrict__ ptab, BodiesV B, const float4* __restrict__ pre_lin,
                             const float4* __restrict__ pre_ang, RowsV R, float* acc_jn, float2* acc_jt,
                             const uint32_t* __restrict__ uf, uint32_t* row_root, const uint8_t* __restrict__ jointed,
                             const float4* __restrict__ last_lin, float4* toi_a, float2* toi_b) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  bool terrain = c_b[k] == 0xFFFFFFFFu;
  uint32_t ai = cbody[c_a[k]], bi = terrain ? 0 : cbody[c_b[k]];
  bool a_aw = B.awake[ai] != 0, b_aw = terrain ? false : B.awake[bi] != 0;
  float inv_a = a_aw ? B.inv_mass[ai] : 0.0f, inv_b = b_aw ? B.inv_mass[bi] : 0.0f;
  m3 IA = inv_a > 0.0f ? ld_m3(B.Iw, ai) : mzero();
  m3 IB = inv_b > 0.0f ? ld_m3(B.Iw, bi) : mzero();
  uint32_t ma = cmat[c_a[k]], mb = terrain ? hf_mat : cmat[c_b[k]];
  const float* pp = ptab + 5 * (ma * 14 + mb);
  float4 cp = c_pt[k], cn = c_n[k];
  f3 point = xyz(cp), n = xyz(cn);
  f3 t1, t2;
  orthonormal_basis(n, &t1, &t2);
  f3 pa = xyz(B.pos[ai]);
  f3 ra = point - pa;
  f3 rb = terrain ? mk3(0, 0, 0) : point - xyz(B.pos[bi]);
  float m_n = eff_mass(inv_a, inv_b, IA, IB, ra, rb, n);
  float m_t1 = eff_mass(inv_a, inv_b, IA, IB, ra, rb, t1);
  float m_t2 = eff_mass(inv_a, inv_b, IA, IB, ra, rb, t2);
  float mu_s = pp[0], mu_k = pp[1], rest = pp[2], sv = rmax(pp[3], 1.0e-4f);
  float pen = cp.w - 0.05f;
  float bias = pen > 0.0f ? rmin(rmax(pen - 0.005f, 0.0f) * (0.05f / dt), 2.0f) : pen / dt;
  // approach at mid-step (:538-544) and the restitution target (:569-588)
  f3 val = xyz(pre_lin[ai]), vaa = xyz(pre_ang[ai]);
  f3 vbl = terrain ? mk3(0, 0, 0) : xyz(pre_lin[bi]), vba = terrain ? mk3(0, 0, 0) : xyz(pre_ang[bi]);
  float v_pre = dot((vbl + cross(vba, rb)) - (val + cross(vaa, ra)), n);
  f3 va = xyz(B.lin[ai]) + cross(xyz(B.ang[ai]), ra);
  f3 vb = terrain ? mk3(0, 0, 0) : xyz(B.lin[bi]) + cross(xyz(B.ang[bi]), rb);
  float v_rel_n = 0.5f * (v_pre + dot(vb - va, n));
  float rbias = 0.0f;
  uint32_t flags = terrain ? RF_TERRAIN : 0u;
  const bool ja = jointed && jointed[ai], jb = jointed && !terrain && jointed[bi];
  if (v_rel_n < -1.0f) {
    rbias = (-rest) * v_rel_n;
    if (!ja && !jb) {  // W6: free bodies bounce at their time of impact (solver.rs:571-587)
      flags |= RF_TOI;
      // each side's normal velocity at the contact from the integrator's start velocities (last
      // step's linear, the start angular) and after this step's forces
      auto at = [&](f3 l, f3 a, f3 r) { return dot(l + cross(a, r), n); };
      float vb0 = 0.0f, vb1 = 0.0f;
      if (!terrain) {
        vb0 = at(xyz(last_lin[bi]), vba, rb);
        vb1 = at(xyz(B.lin[bi]), xyz(B.ang[bi]), rb);
      }
      toi_a[k] = make_float4(-pen, rest, at(xyz(last_lin[ai]), vaa, ra), at(xyz(B.lin[ai]), xyz(B.ang[ai]), ra));
      toi_b[k] = make_float2(vb0, vb1);
    }
  }
  bool wa = inv_a > 0.0f, wb = !terrain && inv_b > 0.0f;
  if (wa) flags |= RF_WA;
  if (wb) flags |= RF_WB;
  // a sleeping side in a joint: read while its joint rows move it, so ordered like a write
  if ((wa || wb) && !wa && ja && B.inv_mass[ai] > 0.0f) flags |= RF_RA;
  if ((wa || wb) && !wb && jb && B.inv_mass[bi] > 0.0f) flags |= RF_RB;
  R.ab[k] = make_uint2(ai, bi);
  R.flags[k] = flags;
  R.inv[k] = make_float2(inv_a, inv_b);
  R.ra[k] = f4(ra, m_n);
  R.rb[k] = f4(rb, m_t1);
  R.n[k] = f4(n, m_t2);
  R.t1[k] = f4(t1, bias);
  R.t2[k] = f4(t2, rbias);
  R.mu[k] = make_float4(mu_s, mu_k, sv, 0.0f);
  R.la[k] = f4(qrot(qconj(asq(B.rot[ai])), point - pa));
  acc_jn[k] = 0.0f;
  acc_jt[k] = make_float2(0.0f, 0.0f);
  row_root[k] = (wa || wb) ? uf_find(const_cast<uint32_t*>(uf), (flags & RF_TA) ? ai : bi) : 0xFFFFFFFFu;
}

// ------------------------------------------------------------------ row math shared by passes
struct Row {
  uint32_t ai, bi, flags;
  float inv_a, inv_b;
  f3 ra, rb, n, t1, t2;
  float m_n, m_t1, m_t2, mu_s, mu_k, sv, bias, rbias;
};
__device__ __forceinline__ Row ld_row(const RowsV& R, uint32_t k) {
  Row r;
  uint2 ab = R.ab[k];
  r.ai = ab.x; r.bi = ab.y; r.flags = R.flags[k];
  float2 iv = R.inv[k]; r.inv_a = iv.x; r.inv_b = iv.y;
  float4 a = R.ra[k], b = R.rb[k], n = R.n[k], t1 = R.t1[k], t2 = R.t2[k], mu = R.mu[k];
  r.ra = xyz(a); r.m_n = a.w; r.rb = xyz(b); r.m_t1 = b.w; r.n = xyz(n); r.m_t2 = n.w;
  r.t1 = xyz(t1); r.bias = t1.w; r.t2 = xyz(t2); r.rbias = t2.w;
  r.mu_s = mu.x; r.mu_k = mu.y; r.sv = mu.z;
  return r;
}
__device__ __forceinline__ f3 rel_vel(const BodiesV& B, const Row& r) {
  f3 va = xyz(B.lin[r.ai]) + cross(xyz(B.ang[r.ai]), r.ra);
  f3 vb = (r.flags & RF_TERRAIN) ? mk3(0, 0, 0) : xyz(B.lin[r.bi]) + cross(xyz(B.ang[r.bi]), r.rb);
  return vb - va;
}
// Bodies::apply_impulse alone (dynamics.rs:193-197): the linear part
__device__ __forceinline__ void lin_impulse(const BodiesV& B, uint32_t i, f3 j) {
  float im = B.inv_mass[i];
  if (im > 0.0f && vfin(j)) { float4 l = B.lin[i]; B.lin[i] = f4(fin_v(xyz(l) + j * im), l.w); }
}
// Bodies::apply_impulse / apply_angular_impulse (dynamics.rs:193-205) with the tick's R I^-1 R^T
__device__ __forceinline__ void body_impulse(const BodiesV& B, uint32_t i, f3 j, f3 tau) {
  float im = B.inv_mass[i];
  if (im > 0.0f && vfin(j)) { float4 l = B.lin[i]; B.lin[i] = f4(fin_v(xyz(l) + j * im), l.w); }
  if (B.inv_mass[i] > 0.0f && vfin(tau)) {
    f3 dw = mvec(ld_m3(B.Iw, i), tau);
    float4 a = B.ang[i];
    B.ang[i] = f4(fin_v(xyz(a) + dw), a.w);
  }
}
// apply_contact_impulse (solver.rs:455-464)
__device__ __forceinline__ void contact_impulse(const BodiesV& B, const Row& r, f3 j) {
  if (r.inv_a > 0.0f) { f3 nj = -j; body_impulse(B, r.ai, nj, cross(r.ra, nj)); }
  if (r.inv_b > 0.0f) body_impulse(B, r.bi, j, cross(r.rb, j));
}
#include "bounce.cuh"
// The friction law mu_k + (mu_s - mu_k) * exp(-(slip / sv)^2). Where mu_s == mu_k and slip / sv is
// a number, exp's value lies in [0, 1], so (mu_s - mu_k) * exp(...) has the bits of
// (mu_s - mu_k) * 0 (+0, or NaN for infinite coefficients): the law is evaluated without the
// division and the exp, with the same result.
__device__ __forceinline__ bool ratio_is_nan(float a, float b) {
  return isnan(a) || isnan(b) || (a == 0.0f && b == 0.0f) || (isinf(a) && isinf(b));
}
__device__ __forceinline__ float mu_law(float mu_s, float mu_k, float sv, float slip) {
  if (mu_s == mu_k && !ratio_is_nan(slip, sv)) return mu_k + (mu_s - mu_k) * 0.0f;
  float t = slip / sv;
  return mu_k + (mu_s - mu_k) * exp_rp(-(t * t));
}
__device__ __forceinline__ float mu_dynamic(const Row& r, float slip) {  // solver.rs:429-431
  return mu_law(r.mu_s, r.mu_k, r.sv, slip);
}
// Warm start of one matched row (solver.rs:749-760)
__device__ __forceinline__ void warm_apply(const BodiesV& B, const Row& r, uint32_t k, float4 ea, float4 eb,
                                           float* acc_jn, float2* acc_jt) {
  float jn = ea.w;
  f3 jt = xyz(eb);
  acc_jn[k] = jn;
  f3 imp = r.n * jn;
  f3 v = rel_vel(B, r);
  float a = dot(v, r.t1), b = dot(v, r.t2);
  float mu = mu_dynamic(r, sqrtf(a * a + b * b));
  f3 t = clamp_length_max(mk3(dot(jt, r.t1), dot(jt, r.t2), 0.0f), mu * jn);
  acc_jt[k] = make_float2(t.x, t.y);
  imp = imp + ((r.t1 * t.x) + (r.t2 * t.y));
  contact_impulse(B, r, imp);
}
// One Gauss-Seidel update of a contact row (solver.rs:857-878); returns the row's residual.
__device__ __forceinline__ float pgs_row(const BodiesV& B, const Row& r, uint32_t k, float* acc_jn, float2* acc_jt) {
  float v_rel_n = dot(rel_vel(B, r), r.n);
  float jn_raw = (r.bias - v_rel_n) * r.m_n;
  float old_jn = acc_jn[k];
  float new_jn = rmax(old_jn + jn_raw, 0.0f);
  acc_jn[k] = new_jn;
  contact_impulse(B, r, r.n * (new_jn - old_jn));
  f3 vf = rel_vel(B, r);
  float vt1 = dot(vf, r.t1), vt2 = dot(vf, r.t2);
  float slip = sqrtf(vt1 * vt1 + vt2 * vt2);
  float mu = mu_dynamic(r, slip);
  float2 ot = acc_jt[k];
  f3 old_t = mk3(ot.x, ot.y, 0.0f);
  f3 new_t = clamp_length_max(old_t - mk3(vt1 * r.m_t1, vt2 * r.m_t2, 0.0f), mu * new_jn);
  acc_jt[k] = make_float2(new_t.x, new_t.y);
  f3 d = new_t - old_t;
  contact_impulse(B, r, (r.t1 * d.x) + (r.t2 * d.y));
  float res = 0.0f;
  if (r.m_n > 0.0f) res = rmax(res, fabsf(new_jn - old_jn) / r.m_n);
  if (r.m_t1 > 0.0f) res = rmax(res, fabsf(d.x) / r.m_t1);
  if (r.m_t2 > 0.0f) res = rmax(res, fabsf(d.y) / r.m_t2);
  return res;
}

// The unclamped joint impulse (solver.rs:821-830): a rigid row drives v to the target, a damper row
// (gamma = 1 / (damping dt) > 0) drives v + gamma lam to it.
__device__ __forceinline__ float joint_lam(float old, float target, float v, float gamma, float m_eff) {
  return gamma == 0.0f ? old + (target - v) * m_eff : old + ((target - v) - gamma * old) * m_eff;
}
// A joint velocity row on the global body arrays (the warp kernel of the largest islands).
__device__ __forceinline__ void joint_apply_glob(const BodiesV& B, const Row& r, float lam) {
  f3 p = r.n * lam;
  if (r.flags & RF_JANG) {
    f3 t = -p;
    if (r.inv_a > 0.0f && B.inv_mass[r.ai] > 0.0f && vfin(t)) {
      float4 a = B.ang[r.ai];
      B.ang[r.ai] = f4(fin_v(xyz(a) + mvec(ld_m3(B.Iw, r.ai), t)), a.w);
    }
    if (r.inv_b > 0.0f && B.inv_mass[r.bi] > 0.0f && vfin(p)) {
      float4 a = B.ang[r.bi];
      B.ang[r.bi] = f4(fin_v(xyz(a) + mvec(ld_m3(B.Iw, r.bi), p)), a.w);
    }
  } else {
    if (r.inv_a > 0.0f) { f3 nj = -p; body_impulse(B, r.ai, nj, cross(r.ra, nj)); }
    if (r.inv_b > 0.0f) body_impulse(B, r.bi, p, cross(r.rb, p));
  }
}
// The original distance row (solver.rs:793-817) on the global arrays: returns the impulse.
__device__ __forceinline__ float legacy_row_glob(const BodiesV& B, const Row& r) {
  float v_rel = dot(xyz(B.lin[r.bi]) - xyz(B.lin[r.ai]), r.n);
  float j_mag = -(v_rel + r.bias) / r.m_t1;
  lin_impulse(B, r.ai, (-r.n) * j_mag);
  lin_impulse(B, r.bi, r.n * j_mag);
  return j_mag;
}
__device__ __forceinline__ float joint_row_glob(const BodiesV& B, const Row& r, uint32_t k, float* acc_jn) {
  if (r.flags & RF_JNULL) return 0.0f;
  if (r.flags & RF_JLEG) return fabsf(legacy_row_glob(B, r)) / r.m_n;
  f3 va, vb;
  if (r.flags & RF_JANG) { va = xyz(B.ang[r.ai]); vb = xyz(B.ang[r.bi]); }
  else {
    va = xyz(B.lin[r.ai]) + cross(xyz(B.ang[r.ai]), r.ra);
    vb = xyz(B.lin[r.bi]) + cross(xyz(B.ang[r.bi]), r.rb);
  }
  float v = dot(vb - va, r.n);
  float old = acc_jn[k];
  float nw = clampf(joint_lam(old, r.bias, v, r.t1.z, r.m_n), r.mu_s, r.mu_k);
  acc_jn[k] = nw;
  if (nw != old) joint_apply_glob(B, r, nw - old);
  return fabsf(nw - old) / r.m_n;
}

// ------------------------------------------------------------------ warm matching
// Keys (solver.rs:720-726): (body A, body B or u32::MAX, ordinal A, ordinal B); every body has
// one collider, so both ordinals are 0.
__device__ __forceinline__ uint4 row_key(uint32_t a, bool terrain, uint32_t b) {
  return terrain ? make_uint4(a, 0xFFFFFFFFu, 0u, 0u) : make_uint4(a, b, 0u, 0u);
}
__device__ __forceinline__ bool key_lt(uint4 a, uint4 b) {
  if (a.x != b.x) return a.x < b.x;
  if (a.y != b.y) return a.y < b.y;
  if (a.z != b.z) return a.z < b.z;
  return a.w < b.w;
}
__device__ __forceinline__ bool key_eq(uint4 a, uint4 b) { return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w; }
__device__ __forceinline__ uint32_t key_lower_bound(const uint4* keys, uint32_t n, uint4 k) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) { uint32_t mid = (lo + hi) >> 1; if (key_lt(keys[mid], k)) lo = mid + 1; else hi = mid; }
  return lo;
}
// One thread per run of contacts sharing a key: the nearest unused cached anchor within 1 cm,
// lowest index on ties (solver.rs:733-748). Records the entry index per contact (-1: cold).
__global__ void k_warm_match(uint32_t nc, const uint2* __restrict__ ab, const uint32_t* __restrict__ flags,
                             const float4* __restrict__ la, const uint4* __restrict__ wkey, const float4* __restrict__ wa,
                             uint32_t nw, int* wm_idx, uint32_t* n_matched, uint32_t* err) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  uint2 x = ab[k];
  uint4 key = row_key(x.x, flags[k] & RF_TERRAIN, x.y);
  if (k > 0) {
    uint2 y = ab[k - 1];
    if (key_eq(row_key(y.x, flags[k - 1] & RF_TERRAIN, y.y), key)) return;  // not the run's first
  }
  uint32_t e0 = key_lower_bound(wkey, nw, key), e1 = e0;
  while (e1 < nw && key_eq(wkey[e1], key)) e1++;
  unsigned long long used = 0ull;
  if (e1 - e0 > 64) { atomicOr(err, 2u); e1 = e0 + 64; }
  const float tol2 = 0.01f * 0.01f;
  uint32_t matched = 0;
  for (uint32_t c = k; c < nc; ++c) {
    if (c > k) {
      uint2 z = ab[c];
      if (!key_eq(row_key(z.x, flags[c] & RF_TERRAIN, z.y), key)) break;
    }
    f3 anchor = xyz(la[c]);
    int best = -1; float bd = 0.0f;
    for (uint32_t e = e0; e < e1; ++e) {
      if (used & (1ull << (e - e0))) continue;
      float d = len2(xyz(wa[e]) - anchor);
      if (d <= tol2 && (best < 0 || d < bd)) { best = (int)e; bd = d; }
    }
    if (best >= 0) { used |= 1ull << (best - (int)e0); matched++; }
    wm_idx[c] = best;
  }
  if (matched) atomicAdd(n_matched, matched);
}
// Matched rows with no movable body: their impulses are set, nothing moves (solver.rs:749-760).
__global__ void k_warm_unscheduled(uint32_t nc, RowsV R, BodiesV B, const int* __restrict__ wm_idx,
                                   const float4* __restrict__ wa, const float4* __restrict__ wb, float* acc_jn,
                                   float2* acc_jt) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  uint32_t f = R.flags[k];
  if (f & (RF_WA | RF_WB)) return;
  int e = wm_idx[k];
  if (e < 0) return;
  Row r = ld_row(R, k);
  warm_apply(B, r, k, wa[e], wb[e], acc_jn, acc_jt);
}

// ------------------------------------------------------------------ schedules
// Greedy level schedule (solver.rs:621-642) in parallel. In the serial order `ord_in`, a row's
// level is one more than the level of the previous row writing any of its bodies (0 if none):
// level(s) = max over its predecessors p of level(p) + 1. Predecessors come from a stable sort of
// (body, position) entries; the levels are then the fixed point of that recurrence on the
// predecessor DAG, reached by monotone relaxation from 0 (after k passes every row whose longest
// predecessor chain has length <= k is exact; an acyclic graph converges in depth + 1 passes).
// Each row is one position s in ord_in; positions of one island are contiguous.
// Joint units (t1 non-null): a joint's rows after its first are scheduled with it -- same level,
// right after it (one thread runs them in order) -- so they take no body entries and lead[s] is the
// distance back to the joint's first row (0 for every other row).
__global__ void k_level_entries(uint32_t n, const uint32_t* __restrict__ ord_in, const uint2* __restrict__ ab,
                                const uint32_t* __restrict__ flags, const float4* __restrict__ t1, uint32_t* key,
                                uint32_t* val, uint32_t* lead) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t r = ord_in[s];
  uint2 x = ab[r];
  uint32_t f = flags[r];
  const bool tail = t1 && (f & RF_JOINT) && !(f & RF_JFIRST);
  key[2 * s] = (!tail && (f & RF_TA)) ? x.x : 0xFFFFFFFFu;
  key[2 * s + 1] = (!tail && (f & RF_TB)) ? x.y : 0xFFFFFFFFu;
  val[2 * s] = 2 * s;
  val[2 * s + 1] = 2 * s + 1;
  if (lead) lead[s] = tail ? (uint32_t)t1[r].y : 0u;
}
// entries sorted by body (stable): the previous entry of the same body is the predecessor
__global__ void k_level_preds(uint32_t m, const uint32_t* __restrict__ key, const uint32_t* __restrict__ val,
                              uint32_t* pred) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m) return;
  uint32_t b = key[e];
  if (b == 0xFFFFFFFFu) return;
  pred[val[e]] = (e > 0 && key[e - 1] == b) ? (val[e - 1] >> 1) : 0xFFFFFFFFu;
}
// One warp per island: lanes own contiguous chunks of the island's positions and sweep them in
// order (so chains inside a chunk settle in one pass) until a pass changes nothing.
__global__ void k_level_relax(uint32_t nisl, const uint32_t* __restrict__ isl_start, const uint32_t* __restrict__ isl_cnt,
                              const uint32_t* __restrict__ ord_in, const uint32_t* __restrict__ pred,
                              const uint32_t* __restrict__ lead, uint32_t* level, unsigned long long* key_out,
                              uint32_t* nlev, uint32_t* row_level, uint32_t* err) {
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t lane = threadIdx.x & 31;
  if (warp >= nisl) return;
  uint32_t s0 = isl_start[warp], n = isl_cnt[warp];
  uint32_t chunk = (n + 31) / 32;
  uint32_t a = s0 + lane * chunk, z = a + chunk;
  if (z > s0 + n) z = s0 + n;
  for (uint32_t s = a; s < z; ++s) level[s] = 0;
  __syncwarp();
  volatile uint32_t* vl = level;
  uint32_t passes = 0;
  while (true) {
    bool changed = false;
    for (uint32_t s = a; s < z; ++s) {
      uint32_t p0 = pred[2 * s], p1 = pred[2 * s + 1];
      uint32_t L = 0;
      if (lead && lead[s]) L = vl[s - lead[s]];  // a joint's later row: its first row's level
      if (p0 != 0xFFFFFFFFu) { uint32_t v = vl[p0] + 1; if (v > L) L = v; }
      if (p1 != 0xFFFFFFFFu) { uint32_t v = vl[p1] + 1; if (v > L) L = v; }
      if (L != vl[s]) { vl[s] = L; changed = true; }
    }
    __syncwarp();
    if (!__any_sync(0xffffffffu, changed)) break;
    if (++passes > n + 2) { if (lane == 0) atomicOr(err, 4u); break; }  // cannot happen on a DAG
  }
  uint32_t mx = 0;
  for (uint32_t s = a; s < z; ++s) {
    uint32_t L = vl[s];
    key_out[s] = ((unsigned long long)warp << 32) | L;
    if (row_level) row_level[ord_in[s]] = L;
    if (L + 1 > mx) mx = L + 1;
  }
  for (int o = 16; o > 0; o >>= 1) { uint32_t t = __shfl_xor_sync(0xffffffffu, mx, o); if (t > mx) mx = t; }
  if (lane == 0) nlev[warp] = mx;
}
// Coloured order (worlds without joints): one warp per group walks its levels in order, and each
// row of a level takes the smallest colour that no already coloured row writing one of its bodies
// holds (first fit; 128 colours per body, bits in col_mask). The rows of one level share no written
// body, so the warp colours them at once, and the result is the sequential first fit in level
// order. A group where some row finds no free colour keeps its levels (flag over), and so does a
// group of one island (g >= g_small) whose colours are no fewer than its
// levels if it has more than 32 rows. Output: the (group, colour) key of every schedule position and
// the group's step count.
__global__ void k_colour_levels(uint32_t ng, uint32_t g_small, const uint32_t* __restrict__ ord, const uint32_t* __restrict__ lvl_off,
                                const uint32_t* __restrict__ lvl_start, const uint32_t* __restrict__ nlev,
                                const uint2* __restrict__ ab, const uint32_t* __restrict__ flags, uint4* mask,
                                unsigned long long* key_out, uint32_t* ncol) {
  const uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  if (g >= ng) return;
  const uint32_t off = lvl_off[g], nl = nlev[g];
  bool over = false;
  uint32_t mx = 0;
  for (uint32_t L = 0; L < nl; ++L) {
    const uint32_t s1 = lvl_start[off + L + 1];
    for (uint32_t s = lvl_start[off + L] + lane; s < s1; s += 32u) {
      const uint32_t r = ord[s], f = flags[r];
      const uint2 x = ab[r];
      const bool ta = (f & RF_TA) != 0, tb = (f & RF_TB) != 0;
      uint4 m = make_uint4(0u, 0u, 0u, 0u), ma = m, mb = m;
      if (ta) ma = mask[x.x];
      if (tb) mb = mask[x.y];
      m = make_uint4(ma.x | mb.x, ma.y | mb.y, ma.z | mb.z, ma.w | mb.w);
      uint32_t c = 0xFFFFFFFFu;
      if (~m.x) c = __ffs(~m.x) - 1;
      else if (~m.y) c = 32u + __ffs(~m.y) - 1;
      else if (~m.z) c = 64u + __ffs(~m.z) - 1;
      else if (~m.w) c = 96u + __ffs(~m.w) - 1;
      if (c == 0xFFFFFFFFu) {
        over = true;
      } else {
        const uint32_t bit = 1u << (c & 31u), w = c >> 5;
        if (ta) { (&ma.x)[w] |= bit; mask[x.x] = ma; }
        if (tb) { (&mb.x)[w] |= bit; mask[x.y] = mb; }
        if (c + 1u > mx) mx = c + 1u;
      }
      key_out[s] = ((unsigned long long)g << 32) | c;
    }
    __syncwarp();  // this level's colours reach the masks before the next level reads them
  }
  over = __any_sync(0xffffffffu, over);
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (g >= g_small && lvl_start[off + nl] - lvl_start[off] > 32u && mx >= nl) over = true;
  if (over) {
    for (uint32_t L = 0; L < nl; ++L)
      for (uint32_t s = lvl_start[off + L] + lane; s < lvl_start[off + L + 1]; s += 32u)
        key_out[s] = ((unsigned long long)g << 32) | L;
  }
  if (lane == 0) ncol[g] = over ? nl : mx;
}
// The residual histogram over the solve islands from each island's last-sweep residual (bits).
__global__ void k_res_hist(uint32_t nisl, const uint32_t* __restrict__ isl_final, uint32_t* stats) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nisl) atomicAdd(&stats[STAT_RES_HIST + res_bin(__uint_as_float(isl_final[i]))], 1u);
}
__global__ void k_row_key_level(uint32_t n, const uint32_t* __restrict__ ord, const unsigned long long* __restrict__ keys,
                                uint32_t* row_level) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) row_level[ord[s]] = (uint32_t)keys[s];
}
__global__ void k_plus1(uint32_t n, const uint32_t* __restrict__ a, uint32_t* b) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i] + 1;
}
// Level start positions per island (+ a sentinel at the island's end), and the global
// per-level histogram (solver.rs:684-687's last_max_batch).
__global__ void k_level_starts(uint32_t n, const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ lvl_off,
                               const uint32_t* __restrict__ nlev, const uint32_t* __restrict__ isl_start,
                               const uint32_t* __restrict__ isl_cnt, uint32_t* lvl_start, uint32_t* hist) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  unsigned long long k = keys[s];
  uint32_t isl = (uint32_t)(k >> 32), L = (uint32_t)k;
  if (s == 0 || keys[s - 1] != k) lvl_start[lvl_off[isl] + L] = s;
  if (s == isl_start[isl]) lvl_start[lvl_off[isl] + nlev[isl]] = isl_start[isl] + isl_cnt[isl];
  if (hist) atomicAdd(&hist[L], 1u);
}
__global__ void k_gather_u32(uint32_t n, const uint32_t* __restrict__ idx, const uint32_t* __restrict__ src, uint32_t* dst) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

struct Sched { uint32_t* ord; uint32_t* lvl_off; uint32_t* lvl_start; uint32_t* nlev; };

// Warm start, joints (solver.rs:699-712): every joint row's clamped previous impulse, applied when
// not 0, before any contact's warm start -- the reference's order (all joints, then the contacts,
// whose friction clamp reads the bodies' velocities after the joints' impulses). One warp per solve
// group walks its levels: the joint rows of a body come in joint order.
__global__ void k_joint_warm(uint32_t ng, uint32_t nc, Sched S, RowsV R, BodiesV B, float* acc_jn) {
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= ng) return;
  uint32_t off = S.lvl_off[warp], nl = S.nlev[warp];
  for (uint32_t L = 0; L < nl; ++L) {
    uint32_t s0 = S.lvl_start[off + L], s1 = S.lvl_start[off + L + 1];
    for (uint32_t s = s0 + lane; s < s1; s += 32) {
      uint32_t k = S.ord[s];
      if (k < nc || (R.flags[k] & (RF_JWARM | RF_JFIRST)) != (RF_JWARM | RF_JFIRST)) continue;
      const uint32_t cnt = (uint32_t)R.t1[k].x;  // the unit's rows follow its first, in order
      for (uint32_t q = 0; q < cnt; ++q) {
        uint32_t kq = S.ord[s + q];
        Row r = ld_row(R, kq);
        acc_jn[kq] = r.t2.x;
        if (r.t2.x != 0.0f) joint_apply_glob(B, r, r.t2.x);
      }
    }
    __syncwarp();
  }
}


// ------------------------------------------------------------------ island passes (warp per island)
__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
// Warm start application, then the velocity sweeps (solver.rs:717-915).
__global__ void k_vel_solve(uint32_t nisl, uint32_t nc, Sched S, RowsV R, BodiesV B, float* acc_jn, float2* acc_jt,
                            const int* __restrict__ wm_idx, const float4* __restrict__ wa, const float4* __restrict__ wb,
                            int iters, float tol, uint32_t* stats, const uint32_t* __restrict__ g_class,
                            const uint32_t* __restrict__ glist, const uint32_t* __restrict__ row_islid,
                            uint32_t* isl_final) {
  uint32_t wi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (wi >= nisl) return;
  uint32_t warp = glist[wi];  // nisl: the number of listed groups
  if (g_class[warp] != 2u) return;
  uint32_t off = S.lvl_off[warp], nl = S.nlev[warp];
  for (uint32_t L = 0; L < nl; ++L) {
    uint32_t s0 = S.lvl_start[off + L], s1 = S.lvl_start[off + L + 1];
    for (uint32_t s = s0 + lane; s < s1; s += 32) {
      uint32_t k = S.ord[s];
      if (k >= nc) continue;  // joint rows: started by k_joint_warm
      int e = wm_idx[k];
      if (e >= 0) { Row r = ld_row(R, k); warm_apply(B, r, k, wa[e], wb[e], acc_jn, acc_jt); }
    }
    __syncwarp();
  }
  int it = 0;
  float resid = 0.0f;
  while (it < iters) {
    resid = 0.0f;
    for (uint32_t L = 0; L < nl; ++L) {
      uint32_t s0 = S.lvl_start[off + L], s1 = S.lvl_start[off + L + 1];
      for (uint32_t s = s0 + lane; s < s1; s += 32) {
        uint32_t k = S.ord[s];
        Row r = ld_row(R, k);
        if (k >= nc) {  // a joint unit: its first row runs all its rows in order
          if (!(r.flags & RF_JFIRST)) continue;
          const uint32_t cnt = (uint32_t)r.t1.x;
          for (uint32_t q = 0; q < cnt; ++q) {
            uint32_t kq = S.ord[s + q];
            resid = rmax(resid, joint_row_glob(B, q ? ld_row(R, kq) : r, kq, acc_jn));
          }
          continue;
        }
        resid = rmax(resid, pgs_row(B, r, k, acc_jn, acc_jt));
      }
      __syncwarp();
    }
    it++;
    resid = warp_max(resid);
    if (tol > 0.0f && resid <= tol) break;
  }
  if (lane == 0) {
    const uint32_t nrows = S.lvl_start[off + nl] - S.lvl_start[off];
    atomicAdd(&stats[STAT_ROWSWEEPS], nrows * (uint32_t)it);
    atomicMax(&stats[STAT_SWEEPS], (uint32_t)it);
    atomicMax(&stats[STAT_RESID], fbits(resid));
    isl_final[row_islid[S.ord[S.lvl_start[off]]]] = fbits(resid);  // the group is one island
    if (tol > 0.0f && !(resid <= tol)) {
      atomicAdd(&stats[STAT_ISLANDS_CAPPED], 1u);
      atomicAdd(&stats[STAT_ROWS_CAPPED], nrows);
    }
  }
}
// Shock propagation (solver.rs:964-993): rows in (1e-6 height key, index) order, the lower body
// of a two-body row frozen for its update.
__global__ void k_vel_shock(uint32_t nisl, Sched S, RowsV R, BodiesV B, f3 up, float* acc_jn) {
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= nisl) return;
  uint32_t off = S.lvl_off[warp], nl = S.nlev[warp];
  for (uint32_t L = 0; L < nl; ++L) {
    uint32_t s0 = S.lvl_start[off + L], s1 = S.lvl_start[off + L + 1];
    for (uint32_t s = s0 + lane; s < s1; s += 32) {
      uint32_t k = S.ord[s];
      Row r = ld_row(R, k);
      if (r.flags & RF_JOINT) continue;
      m3 IA = r.inv_a > 0.0f ? ld_m3(B.Iw, r.ai) : mzero();
      m3 IB = r.inv_b > 0.0f ? ld_m3(B.Iw, r.bi) : mzero();
      if (r.inv_a > 0.0f && r.inv_b > 0.0f) {
        if (dot(xyz(B.pos[r.ai]), up) < dot(xyz(B.pos[r.bi]), up)) { r.inv_a = 0.0f; IA = mzero(); }
        else { r.inv_b = 0.0f; IB = mzero(); }
        r.m_n = eff_mass(r.inv_a, r.inv_b, IA, IB, r.ra, r.rb, r.n);
      }
      float v = dot(rel_vel(B, r), r.n);
      float old = acc_jn[k];
      float nw = rmax(old + (r.bias - v) * r.m_n, 0.0f);
      acc_jn[k] = nw;
      contact_impulse(B, r, r.n * (nw - old));
    }
    __syncwarp();
  }
}
// Shock keys (1e-6 units of the lower body's height; terrain rows -inf) as order-preserving u64.
__global__ void k_shock_keys(uint32_t n, const uint32_t* __restrict__ rows, const uint2* __restrict__ ab,
                             const uint32_t* __restrict__ flags, const float4* __restrict__ pos, f3 up,
                             unsigned long long* keys) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t k = rows[i];
  uint2 x = ab[k];
  float h = (flags[k] & RF_TERRAIN) ? -INFINITY : rmin(dot(xyz(pos[x.x]), up), dot(xyz(pos[x.y]), up));
  long long s = sort_key6(h);
  keys[i] = (unsigned long long)s ^ 0x8000000000000000ull;
}

// Contact load flags (solver.rs:1248-1256), impulse write-back (:1268-1270), W6 rows counted.
__global__ void k_after_solve(uint32_t nc, RowsV R, const float* __restrict__ acc_jn, const float2* __restrict__ acc_jt,
                              uint8_t* loaded, float4* c_n, uint32_t* stats) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  uint2 x = R.ab[k];
  uint32_t f = R.flags[k];
  float jn = acc_jn[k];
  float2 jt = acc_jt[k];
  if (jn > 0.0f || jt.x != 0.0f || jt.y != 0.0f) {
    loaded[x.x] = 1;
    if (!(f & RF_TERRAIN)) loaded[x.y] = 1;
  }
  c_n[k].w = jn;
  (void)stats;
}

// ------------------------------------------------------------------ warm cache rebuild
// solver.rs:917-944: the rows' impulses as the sweeps left them, keyed, in contact order; then
// the old entries of pairs where neither body is awake and dynamic (and still alive).
__global__ void k_warm_new_flags(uint32_t nc, RowsV R, const float* __restrict__ acc_jn, const float2* __restrict__ acc_jt,
                                 uint32_t* flag) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  float2 t = acc_jt[k];
  f3 jt = (xyz(R.t1[k]) * t.x) + (xyz(R.t2[k]) * t.y);
  flag[k] = (acc_jn[k] == 0.0f && vzero(jt)) ? 0u : 1u;
}
__global__ void k_warm_new_write(uint32_t nc, RowsV R, const float* __restrict__ acc_jn, const float2* __restrict__ acc_jt,
                                 const uint32_t* __restrict__ flag, const uint32_t* __restrict__ off,
                                 const uint32_t* __restrict__ okept_cnt_ptr, const uint4* __restrict__ okey, uint32_t n_okept,
                                 uint4* nk, float4* na, float4* nbv) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc || !flag[k]) return;
  uint2 x = R.ab[k];
  uint4 key = row_key(x.x, R.flags[k] & RF_TERRAIN, x.y);
  float2 t = acc_jt[k];
  f3 jt = (xyz(R.t1[k]) * t.x) + (xyz(R.t2[k]) * t.y);
  uint32_t pos = off[k] + key_lower_bound(okey, n_okept, key);
  nk[pos] = key;
  na[pos] = f4(xyz(R.la[k]), acc_jn[k]);
  nbv[pos] = f4(jt);
  (void)okept_cnt_ptr;
}
__device__ __forceinline__ bool idle_body(uint32_t b, const uint8_t* alive, const uint8_t* dyn, const uint8_t* awake, uint32_t nb) {
  if (b == 0xFFFFFFFFu) return true;
  if (b >= nb || !alive[b]) return false;
  return !dyn[b] || !awake[b];
}
__global__ void k_warm_old_flags(uint32_t nw, const uint4* __restrict__ wk, const uint4* __restrict__ newk, uint32_t n_new,
                                 const uint8_t* __restrict__ alive, const uint8_t* __restrict__ dyn,
                                 const uint8_t* __restrict__ awake, uint32_t nb, uint8_t* flag) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nw) return;
  uint4 k = wk[e];
  bool keep = idle_body(k.x, alive, dyn, awake, nb) && idle_body(k.y, alive, dyn, awake, nb);
  if (keep) {
    uint32_t p = key_lower_bound(newk, n_new, k);
    if (p < n_new && key_eq(newk[p], k)) keep = false;
  }
  flag[e] = keep ? 1 : 0;
}

// ------------------------------------------------------------------ stage 4: ballistic + integration
__global__ void k_constrained(uint32_t nc, const uint32_t* __restrict__ c_a, const uint32_t* __restrict__ c_b,
                              const uint32_t* __restrict__ cbody, uint8_t* constrained) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  constrained[cbody[c_a[k]]] = 1;
  if (c_b[k] != 0xFFFFFFFFu) constrained[cbody[c_b[k]]] = 1;
}
__global__ void k_ballistic_init(uint32_t nb, const uint8_t* __restrict__ constrained, const uint8_t* __restrict__ loaded,
                                 const uint8_t* __restrict__ jointed, uint8_t* ballistic) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) ballistic[i] = (!constrained[i] || (!(jointed && jointed[i]) && !loaded[i])) ? 1 : 0;
}
// step.rs:180-206 per contact, on the solve schedule. Flags of bodies that can't move are read
// at their initial value and never written: for those last_lin_vel equals the velocity, so
// their averaged motion equals their velocity, and their flag changes no movable body's outcome.
__global__ void k_ballistic(uint32_t nisl, Sched S, RowsV R, BodiesV B, const float4* __restrict__ c_pt,
                            const float4* __restrict__ c_n, const float4* __restrict__ last_lin, float dt,
                            uint8_t* ballistic) {
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= nisl) return;
  uint32_t off = S.lvl_off[warp], nl = S.nlev[warp];
  for (uint32_t L = 0; L < nl; ++L) {
    uint32_t s0 = S.lvl_start[off + L], s1 = S.lvl_start[off + L + 1];
    for (uint32_t s = s0 + lane; s < s1; s += 32) {
      uint32_t k = S.ord[s];
      uint2 x = R.ab[k];
      uint32_t f = R.flags[k];
      if (f & RF_JOINT) continue;
      bool hb = !(f & RF_TERRAIN);
      uint32_t a = x.x, b = x.y;
      bool ba = ballistic[a] != 0, bb = hb ? ballistic[b] != 0 : false;
      if (!ba && (!hb || !bb)) continue;
      f3 point = xyz(c_pt[k]), n = xyz(c_n[k]);
      f3 la = ba ? (xyz(last_lin[a]) + xyz(B.lin[a])) * 0.5f : xyz(B.lin[a]);
      f3 wa = xyz(B.ang[a]);
      f3 ra = point - xyz(B.pos[a]);
      f3 lb = mk3(0, 0, 0), wb = mk3(0, 0, 0), rb = mk3(0, 0, 0);
      if (hb) { lb = bb ? (xyz(last_lin[b]) + xyz(B.lin[b])) * 0.5f : xyz(B.lin[b]); wb = xyz(B.ang[b]); rb = point - xyz(B.pos[b]); }
      float approach = dot((lb + cross(wb, rb)) - (la + cross(wa, ra)), n);
      f3 vbl = hb ? xyz(B.lin[b]) : mk3(0, 0, 0), vba = hb ? xyz(B.ang[b]) : mk3(0, 0, 0);
      float v_end = dot((vbl + cross(vba, rb)) - (xyz(B.lin[a]) + cross(xyz(B.ang[a]), ra)), n);
      float s0v = -(c_pt[k].w - 0.05f);
      if (s0v + (2.0f * v_end) * dt < 0.0f || s0v + approach * dt < 0.0f) {
        if (f & RF_TA) ballistic[a] = 0;
        if (f & RF_TB) ballistic[b] = 0;
      }
    }
    __syncwarp();
  }
}
// Position integration with the gyroscopic midpoint turn (step.rs:208-280), one thread per body.
__global__ void k_integrate(uint32_t nb, BodiesV B, const uint8_t* __restrict__ ballistic,
                            const float4* __restrict__ last_lin, float dt, float4* orig_pos, float4* orig_rot,
                            float4* pred_pos, float4* pred_rot, const uint32_t* __restrict__ w6_ctr,
                            const float4* __restrict__ w6_pl, const float4* __restrict__ w6_pa) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  float4 P = B.pos[i], Q = B.rot[i];
  orig_pos[i] = P; orig_rot[i] = Q;
  pred_pos[i] = P; pred_rot[i] = Q;
  if (!B.dyn[i] || !B.awake[i]) return;
  f3 pos = xyz(P); q4 rot = asq(Q);
  float4 L = B.lin[i], A = B.ang[i];
  f3 vl = xyz(L), va = xyz(A);
  pos = pos + vl * dt;
  if (ballistic[i]) pos = pos + (xyz(last_lin[i]) - vl) * (0.5f * dt);
  if (len2(va) > 0.0f) {
    m3 l = B.inv_mass[i] == 0.0f ? mzero() : world_inertia(rot, ld_m3(B.inv_I, i));
    float det = mdet(l);
    bool has_m = fin(det) && fabsf(det) > 1.0e-20f;
    f3 m = has_m ? mvec(minverse(l), va) : mk3(0, 0, 0);
    q4 start = rot;
    // turn(q, w, h) = normalize(from_axis_angle(w / |w|, |w| h) * q), or q for |w|^2 <= 1e-18
    {
      f3 w = va;
      if (!(len2(w) <= 1.0e-18f)) rot = qnormalize(qmul(qfrom_axis_angle(normalize(w), len(w) * dt), start));
    }
    if (has_m) {
      m3 il = B.inv_mass[i] == 0.0f ? mzero() : ld_m3(B.inv_I, i);
      float mean = ((il.c0.x + il.c1.y) + il.c2.z) / 3.0f;
      m3 dev = msub(il, mdiag(splat(mean)));
      bool principal = len(cross(m, va)) < (1.0e-5f * len(m)) * len(va);
      float gain = principal ? 0.0f : (dt * rmax(rmax(len(dev.c0), len(dev.c1)), len(dev.c2))) * len(m);
      float cq = ceilf(gain / 0.5f);
      long long nn = isnan(cq) ? 0 : (cq <= 0.0f ? 0 : (cq >= 1.0e18f ? 1000000000000000000LL : (long long)cq));
      int n = (int)(nn < 1 ? 1 : (nn > 256 ? 256 : nn));
      float h = dt / (float)n;
      q4 q = start;
      f3 w = va;
      for (int s = 0; s < n; ++s) {
        q4 q0 = q;
        q = len2(w) <= 1.0e-18f ? q0 : qnormalize(qmul(qfrom_axis_angle(normalize(w), len(w) * h), q0));
        f3 we = mvec(world_inertia(q, il), m);
        for (int r = 0; r < 2; ++r) {
          f3 wm = (w + we) * 0.5f;
          q = len2(wm) <= 1.0e-18f ? q0 : qnormalize(qmul(qfrom_axis_angle(normalize(wm), len(wm) * h), q0));
          we = mvec(world_inertia(q, il), m);
        }
        w = we;
      }
      rot = q;
      va = w;
      if (vfin(vl)) B.lin[i] = f4(fin_v(vl), L.w);  // Bodies::set_vel
      if (vfin(va)) B.ang[i] = f4(fin_v(va), A.w);
    }
  }
  // a bounced free body's pseudo-velocity (W6, step.rs:271-277): moves it, never enters its velocity
  if (w6_ctr[w6::C_PON]) {
    const f3 pl = xyz(w6_pl[i]), pa = xyz(w6_pa[i]);
    pos = pos + pl * dt;
    if (len2(pa) > 0.0f) rot = qnormalize(qmul(qfrom_axis_angle(normalize(pa), len(pa) * dt), rot));
  }
  // Bodies::set_pose (dynamics.rs:130-134)
  if (vfin(pos)) P = f4(fin_v(pos), P.w);
  if (qfin(rot)) Q = f4q(fin_q(rot));
  B.pos[i] = P; B.rot[i] = Q;
  pred_pos[i] = P; pred_rot[i] = Q;
}

// ------------------------------------------------------------------ stage 5: position pass
// pos_contacts (step.rs:423-443): body-local anchors at the start-of-step poses. Row k's A anchor
// is R.la (the warm-start anchor, the same expression); B's is computed here.
__global__ void k_pos_anchors(uint32_t nc, RowsV R, const float4* __restrict__ c_pt, const float4* __restrict__ orig_pos,
                              const float4* __restrict__ orig_rot, float4* lb) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  uint32_t f = R.flags[k];
  if (f & RF_TERRAIN) { lb[k] = make_float4(0, 0, 0, 0); return; }
  uint32_t b = R.ab[k].y;
  lb[k] = f4(qrot(qconj(asq(orig_rot[b])), xyz(c_pt[k]) - xyz(orig_pos[b])));
}
// One projection of contact k (step.rs:457-496).
// The projection of one contact (step.rs:447-497) on an accessor of the bodies' state: pose, inverse
// mass and inertia, whether the body moves (dynamic and awake), the split accumulators. The same
// operations in the same order whatever the accessor, so the global-memory and the shared-memory
// passes give the same bits.
template <class Acc>
__device__ __forceinline__ void project_core(Acc& A, uint32_t a, uint32_t b, bool hb, bool shock, f3 up, f3 n,
                                             float4 cp, f3 la, f3 lb) {
  bool am = A.movable(a);
  bool bm = hb && A.movable(b);
  if (shock && am && bm) {
    float ha = dot(A.pos(a), up), hbb = dot(A.pos(b), up);
    if (ha < hbb) am = false; else bm = false;
  }
  float pen0 = cp.w - 0.05f;
  f3 pa_pos = A.pos(a); q4 pa_rot = A.rot(a);
  f3 wa = pa_pos + qrot(pa_rot, la);
  f3 pb_pos = mk3(0, 0, 0); q4 pb_rot = qident();
  f3 wb;
  if (hb) { pb_pos = A.pos(b); pb_rot = A.rot(b); wb = pb_pos + qrot(pb_rot, lb); }
  else wb = xyz(cp);
  float pen = pen0 - dot(wb - wa, n);
  float err = pen - 0.005f;
  if (err <= 0.0f) return;
  f3 ra = wa - pa_pos;
  f3 rb = hb ? wb - pb_pos : mk3(0, 0, 0);
  float ima = am ? A.inv_mass(a) : 0.0f;
  m3 iia = am ? world_inertia(pa_rot, A.inv_I(a)) : mzero();
  float imb = (hb && bm) ? A.inv_mass(b) : 0.0f;
  m3 iib = (hb && bm) ? world_inertia(pb_rot, A.inv_I(b)) : mzero();
  f3 ca = cross(ra, n), cb = cross(rb, n);
  float w = ((ima + imb) + dot(ca, mvec(iia, ca))) + dot(cb, mvec(iib, cb));
  if (w <= 1.0e-9f) return;
  float lambda = err / w;
  // move_body (step.rs:484-491)
  auto move_body = [&](uint32_t id, f3 ppos, q4 prot, float im, const m3& ii, f3 r, f3 j) {
    f3 dth = mvec(ii, cross(r, j));
    A.split_add(id, j * im, dth);
    q4 dq = qscale(qmul(mkq(dth.x, dth.y, dth.z, 0.0f), prot), 0.5f);
    q4 nr = qnormalize(mkq(prot.x + dq.x, prot.y + dq.y, prot.z + dq.z, prot.w + dq.w));
    f3 np = ppos + j * im;
    if (vfin(np)) A.set_pos(id, fin_v(np));
    if (qfin(nr)) A.set_rot(id, fin_q(nr));
  };
  if (am) move_body(a, pa_pos, pa_rot, ima, iia, ra, (-n) * lambda);
  if (hb && bm) move_body(b, pb_pos, pb_rot, imb, iib, rb, n * lambda);
}
// Body state in global memory (bodies by their world index).
struct PosAccGlobal {
  const BodiesV& B;
  float4* split_l;
  float4* split_a;
  __device__ bool movable(uint32_t i) const { return B.inv_mass[i] > 0.0f && B.awake[i]; }
  __device__ f3 pos(uint32_t i) const { return xyz(B.pos[i]); }
  __device__ q4 rot(uint32_t i) const { return asq(B.rot[i]); }
  __device__ float inv_mass(uint32_t i) const { return B.inv_mass[i]; }
  __device__ m3 inv_I(uint32_t i) const { return ld_m3(B.inv_I, i); }
  __device__ void split_add(uint32_t i, f3 dl, f3 da) {
    float4 sl = split_l[i], sa = split_a[i];
    split_l[i] = f4(xyz(sl) + dl);
    split_a[i] = f4(xyz(sa) + da);
  }
  __device__ void set_pos(uint32_t i, f3 p) { float4 P = B.pos[i]; B.pos[i] = f4(p, P.w); }
  __device__ void set_rot(uint32_t i, q4 q) { B.rot[i] = f4q(q); }
};
__device__ __forceinline__ void project_one(const BodiesV& B, const RowsV& R, uint32_t k, bool shock, f3 up,
                                            const float4* __restrict__ c_pt, const float4* __restrict__ c_n,
                                            const float4* __restrict__ lbv, float4* split_l, float4* split_a) {
  uint2 x = R.ab[k];
  uint32_t f = R.flags[k];
  bool hb = !(f & RF_TERRAIN);
  PosAccGlobal A{B, split_l, split_a};
  project_core(A, x.x, x.y, hb, shock, up, xyz(c_n[k]), c_pt[k], xyz(R.la[k]), hb ? xyz(lbv[k]) : mk3(0, 0, 0));
}
// ---- the position pass with its groups on chip (worlds without joints): a block per solve group
// (the packed groups and the single islands the velocity solve keeps on chip) holds its bodies'
// poses, inverse masses and inertias and split accumulators in shared memory, and its rows' body
// indices, anchors, normals and contact points, for all the iterations; bodies a row reads but
// cannot move (static, asleep, or the terrain) are read from global memory, which nothing writes
// during the pass. Same projections, same order (project_core), so the same bits as
// k_pos_iterations.
struct PosLayout {
  uint32_t RC, BC;
  uint32_t o_pos, o_rot, o_sl, o_sa, o_iI, o_im, o_mov, o_ab, o_la, o_lb, o_n, o_cp, o_lvl, bytes;
};
__host__ __device__ inline PosLayout pos_layout(uint32_t RC, uint32_t BC) {
  PosLayout L;
  L.RC = RC; L.BC = BC;
  uint32_t o = 0;
  auto take = [&](uint32_t bytes) { uint32_t a = o; o = (o + bytes + 15u) & ~15u; return a; };
  L.o_pos = take(16u * BC); L.o_rot = take(16u * BC); L.o_sl = take(16u * BC); L.o_sa = take(16u * BC);
  L.o_iI = take(36u * BC); L.o_im = take(4u * BC); L.o_mov = take(BC);
  L.o_ab = take(8u * RC); L.o_la = take(16u * RC); L.o_lb = take(16u * RC); L.o_n = take(16u * RC); L.o_cp = take(16u * RC);
  L.o_lvl = take(4u * (RC + 1u));
  L.bytes = o;
  return L;
}
// A body index of a row: its index in the group, or 0x80000000 | its world index when the row
// only reads it.
struct PosAccShared {
  float4 *s_pos, *s_rot, *s_sl, *s_sa;
  const float* s_iI;
  const float* s_im;
  const uint8_t* s_mov;
  const BodiesV& G;
  __device__ static bool local(uint32_t i) { return !(i & 0x80000000u); }
  __device__ bool movable(uint32_t i) const {
    const uint32_t g = i & 0x7FFFFFFFu;
    return local(i) ? s_mov[i] != 0 : (G.inv_mass[g] > 0.0f && G.awake[g]);
  }
  __device__ f3 pos(uint32_t i) const { return local(i) ? xyz(s_pos[i]) : xyz(G.pos[i & 0x7FFFFFFFu]); }
  __device__ q4 rot(uint32_t i) const { return local(i) ? asq(s_rot[i]) : asq(G.rot[i & 0x7FFFFFFFu]); }
  __device__ float inv_mass(uint32_t i) const { return local(i) ? s_im[i] : G.inv_mass[i & 0x7FFFFFFFu]; }
  __device__ m3 inv_I(uint32_t i) const { return local(i) ? ld_m3(s_iI, i) : ld_m3(G.inv_I, i & 0x7FFFFFFFu); }
  __device__ void split_add(uint32_t i, f3 dl, f3 da) {  // only a body the group moves
    s_sl[i] = f4(xyz(s_sl[i]) + dl);
    s_sa[i] = f4(xyz(s_sa[i]) + da);
  }
  __device__ void set_pos(uint32_t i, f3 p) { s_pos[i] = f4(p, s_pos[i].w); }
  __device__ void set_rot(uint32_t i, q4 q) { s_rot[i] = f4q(q); }
};
template <int NT>
__global__ void __launch_bounds__(NT) k_pos_onchip(PosLayout Lo, uint32_t n_listed, const uint32_t* __restrict__ glist,
                                                   uint32_t want_class, const uint32_t* __restrict__ g_class,
                                                   const uint32_t* __restrict__ gb_start, const uint32_t* __restrict__ gb_cnt,
                                                   const uint32_t* __restrict__ gb_list, const uint32_t* __restrict__ body_grp,
                                                   const uint32_t* __restrict__ body_local, Sched S, RowsV R, BodiesV G,
                                                   int iters, f3 up, const float4* __restrict__ c_pt,
                                                   const float4* __restrict__ c_n, const float4* __restrict__ lbv,
                                                   float4* split_l, float4* split_a, uint32_t* stats) {
  if (glist && blockIdx.x >= n_listed) return;
  const uint32_t g = glist ? glist[blockIdx.x] : blockIdx.x;
  if (!glist && g >= n_listed) return;
  if (g_class[g] != want_class) return;
  extern __shared__ float4 pos_raw[];
  unsigned char* sb = reinterpret_cast<unsigned char*>(pos_raw);
  float4* pos = reinterpret_cast<float4*>(sb + Lo.o_pos);
  float4* rot = reinterpret_cast<float4*>(sb + Lo.o_rot);
  float4* sl = reinterpret_cast<float4*>(sb + Lo.o_sl);
  float4* sa = reinterpret_cast<float4*>(sb + Lo.o_sa);
  float* iI = reinterpret_cast<float*>(sb + Lo.o_iI);
  float* im = reinterpret_cast<float*>(sb + Lo.o_im);
  uint8_t* mov = sb + Lo.o_mov;
  uint2* ab = reinterpret_cast<uint2*>(sb + Lo.o_ab);
  float4* la = reinterpret_cast<float4*>(sb + Lo.o_la);
  float4* lb = reinterpret_cast<float4*>(sb + Lo.o_lb);
  float4* nn = reinterpret_cast<float4*>(sb + Lo.o_n);
  float4* cp = reinterpret_cast<float4*>(sb + Lo.o_cp);
  uint32_t* lvl = reinterpret_cast<uint32_t*>(sb + Lo.o_lvl);
  const uint32_t tid = threadIdx.x, wid = tid >> 5;
  const uint32_t nbg = gb_cnt[g], b0 = gb_start[g];
  const uint32_t off = S.lvl_off[g], nl = S.nlev[g];
  const uint32_t base = S.lvl_start[off], nr = S.lvl_start[off + nl] - base;
  if (nbg > Lo.BC || nr > Lo.RC || nl > Lo.RC) {  // not reached: the class was chosen by these sizes
    if (tid == 0) atomicOr(&stats[STAT_ERR], 2u);
    return;
  }
  for (uint32_t i = tid; i < nbg; i += NT) {
    const uint32_t b = gb_list[b0 + i];
    pos[i] = G.pos[b]; rot[i] = G.rot[b]; sl[i] = split_l[b]; sa[i] = split_a[b];
    for (int k = 0; k < 9; ++k) iI[9 * i + k] = G.inv_I[9 * (size_t)b + k];
    im[i] = G.inv_mass[b];
    mov[i] = (G.inv_mass[b] > 0.0f && G.awake[b]) ? 1 : 0;
  }
  for (uint32_t i = tid; i < nr; i += NT) {
    const uint32_t k = S.ord[base + i];
    const uint2 x = R.ab[k];
    const bool hb = !(R.flags[k] & RF_TERRAIN);
    const uint32_t a = body_grp[x.x] == g ? body_local[x.x] : (0x80000000u | x.x);
    const uint32_t b = !hb ? 0xFFFFFFFFu : (body_grp[x.y] == g ? body_local[x.y] : (0x80000000u | x.y));
    ab[i] = make_uint2(a, b);
    la[i] = R.la[k];
    lb[i] = hb ? lbv[k] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    nn[i] = c_n[k];
    cp[i] = c_pt[k];
  }
  for (uint32_t L = tid; L <= nl; L += NT) lvl[L] = S.lvl_start[off + L] - base;
  __syncthreads();
  PosAccShared A{pos, rot, sl, sa, iI, im, mov, G};
  auto wide = [&](uint32_t L) { return L < nl && lvl[L + 1] - lvl[L] > 32u; };
  for (int it = 0; it < iters; ++it) {
    for (uint32_t L = 0; L < nl; ++L) {
      for (uint32_t i = lvl[L] + tid; i < lvl[L + 1] && (wid == 0 || wide(L)); i += NT) {
        const uint2 x = ab[i];
        const bool hb = x.y != 0xFFFFFFFFu;
        project_core(A, x.x, x.y, hb, false, up, xyz(nn[i]), cp[i], xyz(la[i]), xyz(lb[i]));
      }
      if (NT == 32 || wide(L) || wide(L + 1)) __syncthreads();
      else __syncwarp();
    }
    __syncthreads();
  }
  for (uint32_t i = tid; i < nbg; i += NT) {
    const uint32_t b = gb_list[b0 + i];
    G.pos[b] = pos[i]; G.rot[b] = rot[i]; split_l[b] = sl[i]; split_a[b] = sa[i];
  }
}

// Position sweeps (step.rs:301-308): each joint's solve (bodies.rs:422-471, SHAKE directions from the
// step's start poses spos / srot) rides on its first velocity row, which the schedule places before
// every later row touching its bodies -- the reference's joints-then-contacts order; joints between
// two frozen (static or sleeping) bodies are skipped. The shock projection has no joints.
// G lanes per group (32 / G groups per warp): narrow groups (a few rows per level, as jointed
// islands are) leave most of a warp idle with one group each. The warp walks the largest level count
// of its groups, lanes of a group that has finished idle; groups never share a body.
// skip: groups of these classes are left to another launch.
template <int G>
__global__ void __launch_bounds__(128) k_pos_iterations(uint32_t n_listed, const uint32_t* __restrict__ glist,
                                                        uint32_t skip, const uint32_t* __restrict__ g_class,
                                                        uint32_t nc, Sched S, RowsV R, BodiesV B, int iters, int shock,
                                                        f3 up, const float4* __restrict__ c_pt,
                                                        const float4* __restrict__ c_n, const float4* __restrict__ lbv,
                                                        float4* split_l, float4* split_a,
                                                        const JointGpu* __restrict__ J, float* jlam,
                                                        const float4* __restrict__ spos, const float4* __restrict__ srot,
                                                        float dt) {
  const uint32_t lane = threadIdx.x & 31, sl = lane % (uint32_t)G;
  const uint32_t slot = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * (32u / G) + lane / (uint32_t)G;
  bool has = slot < n_listed;
  const uint32_t g = has ? (glist ? glist[slot] : slot) : 0u;
  if (has && skip && ((skip >> g_class[g]) & 1u)) has = false;
  const uint32_t off = has ? S.lvl_off[g] : 0u, nl = has ? S.nlev[g] : 0u;
  uint32_t nlw = nl;
  for (int o = 16; o > 0; o >>= 1) nlw = max(nlw, __shfl_xor_sync(0xffffffffu, nlw, o));
  const bool joints_on = !shock && fin(dt) && dt > 0.0f;
  for (int it = 0; it < iters; ++it) {
    for (uint32_t L = 0; L < nlw; ++L) {
      if (L < nl) {
        uint32_t s0 = S.lvl_start[off + L], s1 = S.lvl_start[off + L + 1];
        for (uint32_t s = s0 + sl; s < s1; s += G) {
          uint32_t k = S.ord[s];
          if (k >= nc) {
            if (joints_on && (R.flags[k] & RF_JFIRST)) {
              uint32_t j = __float_as_uint(R.la[k].x);
              const JointGpu& jt = J[j];
              bool fa = !B.dyn[jt.a] || !B.awake[jt.a], fb = !B.dyn[jt.b] || !B.awake[jt.b];
              if (!(fa && fb))
                solve_joint_pos(jt, jlam + 6 * (size_t)j, B, dt, xyz(spos[jt.a]), asq(srot[jt.a]), xyz(spos[jt.b]),
                             asq(srot[jt.b]));
            }
            continue;
          }
          project_one(B, R, k, shock != 0, up, c_pt, c_n, lbv, split_l, split_a);
        }
      }
      __syncwarp();
    }
  }
}
// Restitution (solver.rs:1001-1008) for the rows the W6 passes leave to it -- contacts on jointed
// bodies: one normal update each, in contact order, after the shock pass.
__global__ void k_restitution(uint32_t nisl, uint32_t nc, Sched S, RowsV R, BodiesV B, float* acc_jn) {
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= nisl) return;
  uint32_t off = S.lvl_off[warp], nl = S.nlev[warp];
  for (uint32_t L = 0; L < nl; ++L) {
    uint32_t s0 = S.lvl_start[off + L], s1 = S.lvl_start[off + L + 1];
    for (uint32_t s = s0 + lane; s < s1; s += 32) {
      uint32_t k = S.ord[s];
      if (k >= nc) continue;
      Row r = ld_row(R, k);
      if ((r.flags & RF_TOI) || r.rbias <= 0.0f || acc_jn[k] <= 0.0f) continue;
      float v = dot(rel_vel(B, r), r.n);
      float old = acc_jn[k];
      float nw = rmax(old + (r.rbias - v) * r.m_n, 0.0f);
      acc_jn[k] = nw;
      contact_impulse(B, r, r.n * (nw - old));
    }
    __syncwarp();
  }
}

// ------------------------------------------------------------------ stages 6 and 7
__global__ void k_touching(uint32_t nc, const uint32_t* __restrict__ c_a, const uint32_t* __restrict__ c_b,
                           const float4* __restrict__ c_pt, const uint32_t* __restrict__ cbody, uint8_t* touching) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc || c_b[k] != 0xFFFFFFFFu) return;
  if (c_pt[k].w - 0.05f > -0.005f) touching[cbody[c_a[k]]] = 1;  // no compliant pairs
}
// Velocity from corrections (step.rs:316-376), last velocities (:378-379), sleep (sleep.rs:59-80).
__global__ void k_stage6(uint32_t nb, BodiesV B, const float4* __restrict__ orig_pos, const float4* __restrict__ pred_pos,
                         const float4* __restrict__ pred_rot, const float4* __restrict__ split_l,
                         const float4* __restrict__ split_a, const uint8_t* __restrict__ touching,
                         const uint8_t* __restrict__ jointed, float dt, float4* last_lin, uint8_t* awake,
                         uint16_t* sleep_ticks, const uint8_t* __restrict__ sleep_allowed, uint32_t* stats) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  float4 L = B.lin[i], A = B.ang[i];
  if (B.dyn[i] && awake[i]) {
    f3 vl = xyz(L), va = xyz(A);
    float4 P = B.pos[i];
    f3 np = xyz(P);
    q4 nr = asq(B.rot[i]);
    // split impulse only outside articulations (step.rs:324-329)
    const bool jb = jointed && jointed[i];
    const f3 sl = jb ? mk3(0, 0, 0) : xyz(split_l[i]), sa = jb ? mk3(0, 0, 0) : xyz(split_a[i]);
    f3 d_lin = (np - xyz(pred_pos[i])) - sl;
    if (!vzero(d_lin)) vl = vl + d_lin / dt;
    if (touching[i] && vl.y < 0.0f) {
      vl.y = 0.0f;
      np.y = orig_pos[i].y;
      if (vfin(np)) B.pos[i] = f4(fin_v(np), P.w);
      if (qfin(nr)) B.rot[i] = f4q(fin_q(nr));
    }
    q4 pr = asq(pred_rot[i]);
    // a body of a joint with a rotational velocity drive keeps the angular velocity the motor rows
    // gave it (step.rs:352-366, the motor overwrite): jointed bit 1
    const bool driven = jointed && (jointed[i] & 2u);
    if (!driven && !qeq(nr, pr)) {
      q4 dq = qmul(nr, qconj(pr));
      f3 d_ang = mk3(dq.x, dq.y, dq.z) * 2.0f;
      if (dq.w < 0.0f) d_ang = -d_ang;
      va = va + (d_ang - sa) / dt;
    }
    if (vfin(vl)) L = f4(fin_v(vl), L.w);
    if (vfin(va)) A = f4(fin_v(va), A.w);
    B.lin[i] = L; B.ang[i] = A;
  }
  last_lin[i] = L;
  if (sleep_allowed[i] && awake[i] && B.dyn[i]) {
    if (len2(xyz(L)) < 0.01f && len2(xyz(A)) < 0.01f) {
      uint16_t t = (uint16_t)(sleep_ticks[i] + 1);
      sleep_ticks[i] = t;
      if (t > 30) awake[i] = 0;
    } else {
      sleep_ticks[i] = 0;
    }
  }
}
__global__ void k_count_sleeping(uint32_t n, const uint8_t* __restrict__ awake, uint32_t* stats) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t v = (i < n && awake[i] == 0) ? 1u : 0u;
  v = __reduce_add_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(&stats[STAT_SLEEPING], v);
}

// ------------------------------------------------------------------ solve groups
// Small islands (at most GROUP_ROWS rows) are packed, in order of their row counts, into groups of
// about GROUP_ROWS rows (by the prefix sum of their row counts, so a group holds at most
// 2 * GROUP_ROWS - 1 rows and twice that many bodies); bigger islands form a group alone.
// Islands are independent, so any interleaving of their rows is a valid serial order: a group
// is scheduled and solved exactly like one island. Classes: 3, a packed group, and 10..15, an
// island whose rows and bodies fit in one block's shared memory, are solved by one block with all
// of it on chip; 0, a bigger island, by one CTA with its body velocities on chip and its rows
// streamed through a cp.async double buffer; 2, an island beyond that, by one warp over global
// memory.
// (the row count GROUP_ROWS is a tuning knob, WorldGpu::Tuning::group_rows: 8, 16, 32, 64 or 128)
#define GROUP_ROWS_MAX 128u
// big islands (classes 20..22): bodies and level starts held in shared memory, rows per staged
// chunk (= threads per CTA) -- sized per bucket so that smaller ones share an SM
#define BIG_BUCKETS 3
__constant__ uint32_t c_big_bodies[BIG_BUCKETS] = {1024u, 2048u, 4500u};
__constant__ uint32_t c_big_levels[BIG_BUCKETS] = {2048u, 4096u, 4096u};
static const uint32_t kBigBodies[BIG_BUCKETS] = {1024u, 2048u, 4500u};
static const uint32_t kBigLevels[BIG_BUCKETS] = {2048u, 4096u, 4096u};
#define WG_ROWS(gr) (2u * (gr))    // rows a packed group of group_rows gr can hold
#define WG_BODIES(gr) (4u * (gr))  // bodies those rows can move
// single islands solved with everything on chip, by size bucket (class 10 + bucket): rows and
// bodies held. An island moves at most rows + 1 bodies, so the smaller buckets hold that many;
// the largest one (1152 rows, 768 bodies: 225.8 KB) is sized to the per-block limit.
#define ISLAND_BUCKETS 6
__constant__ uint32_t c_island_rows[ISLAND_BUCKETS] = {128u, 256u, 384u, 512u, 768u, 1152u};
__constant__ uint32_t c_island_bodies[ISLAND_BUCKETS] = {129u, 257u, 385u, 513u, 769u, 768u};
static const uint32_t kIslandRows[ISLAND_BUCKETS] = {128u, 256u, 384u, 512u, 768u, 1152u};
static_assert(ISLAND_BUCKETS + 1 <= WorldGpu::kAux, "a side stream per island bucket and one for the big islands");
static const uint32_t kIslandBodies[ISLAND_BUCKETS] = {129u, 257u, 385u, 513u, 769u, 768u};
__global__ void k_group_flags(uint32_t nisl, uint32_t group_rows, const uint32_t* __restrict__ isl_cnt, uint32_t* small_rows,
                              uint32_t* big) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nisl) return;
  bool small = isl_cnt[i] <= group_rows;
  small_rows[i] = small ? isl_cnt[i] : 0u;
  big[i] = small ? 0u : 1u;
}
__global__ void k_group_of_isl(uint32_t nisl, uint32_t group_rows, const uint32_t* __restrict__ isl_cnt,
                               const uint32_t* __restrict__ small_pre, const uint32_t* __restrict__ big_pre, uint32_t g_small,
                               uint32_t* g_of_isl) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nisl) return;
  g_of_isl[i] = isl_cnt[i] <= group_rows ? small_pre[i] / group_rows : g_small + big_pre[i];
}
// group key of each position of the island-sorted row order (island id = run index)
__global__ void k_group_keys(uint32_t n, const uint32_t* __restrict__ run_flag, const uint32_t* __restrict__ run_pre,
                             const uint32_t* __restrict__ g_of_isl, uint32_t* key) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) key[s] = g_of_isl[run_pre[s] + run_flag[s] - 1];
}
__global__ void k_group_ranges(uint32_t n, const uint32_t* __restrict__ key, uint32_t* start, uint32_t* cnt) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t g = key[s];
  if (s == 0 || key[s - 1] != g) start[g] = s;
  atomicAdd(&cnt[g], 1u);
}
// the group of every body a scheduled row moves (all rows of a body lie in one island)
__global__ void k_body_groups(uint32_t n, const uint32_t* __restrict__ ord, const uint32_t* __restrict__ key,
                              const uint2* __restrict__ ab, const uint32_t* __restrict__ flags, uint32_t* body_grp) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t r = ord[s], g = key[s], f = flags[r];
  uint2 x = ab[r];
  if (f & RF_TA) body_grp[x.x] = g;
  if (f & RF_TB) body_grp[x.y] = g;
}
__global__ void k_flag_grouped(uint32_t nb, const uint32_t* __restrict__ body_grp, uint32_t* flag) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nb) flag[b] = body_grp[b] != 0xFFFFFFFFu;
}
__global__ void k_body_local(uint32_t n, const uint32_t* __restrict__ gkey, const uint32_t* __restrict__ blist,
                             uint32_t* gb_start, uint32_t* gb_cnt, uint32_t* body_local) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  uint32_t g = gkey[p];
  if (p == 0 || gkey[p - 1] != g) gb_start[g] = p;
  atomicAdd(&gb_cnt[g], 1u);
}
__global__ void k_body_local2(uint32_t n, const uint32_t* __restrict__ gkey, const uint32_t* __restrict__ blist,
                              const uint32_t* __restrict__ gb_start, uint32_t* body_local) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) body_local[blist[p]] = p - gb_start[gkey[p]];
}
// Class of every group, and the groups of each class other than 3 listed (in any order: groups
// are independent, so the order they run in changes no result) for launches of exactly them.
__global__ void k_group_class(uint32_t ng, uint32_t g_small, const uint32_t* __restrict__ gb_cnt,
                              const uint32_t* __restrict__ g_cnt, const uint32_t* __restrict__ nlev, uint32_t* cls,
                              uint32_t* cls_cnt, uint32_t* cls_list, uint32_t* stats) {
  uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  uint32_t nbg = gb_cnt[g], nr = g_cnt[g];
  uint32_t c = 3u;
  if (g >= g_small) {
    c = 2u;
    for (int b = BIG_BUCKETS - 1; b >= 0; --b)
      if (nbg <= c_big_bodies[b] && nlev[g] <= c_big_levels[b]) c = 20u + (uint32_t)b;
  }
  if (g >= g_small)
    for (int b = ISLAND_BUCKETS - 1; b >= 0; --b)
      if (nr <= c_island_rows[b] && nbg <= c_island_bodies[b]) c = 10u + (uint32_t)b;
  cls[g] = c;
  if (c != 3u) cls_list[(size_t)c * ng + atomicAdd(&cls_cnt[c], 1u)] = g;  // classes 0..31
  atomicAdd(&stats[c == 2u ? STAT_GROUPS_GLOBAL : STAT_GROUPS_SHARED], 1u);
  atomicMax(&stats[STAT_MAX_GROUP_ROWS], nr);
  atomicMax(&stats[STAT_MAX_GROUP_BODIES], nbg);
}
// Local island index of every scheduled row inside its solve group (islands of a group in island
// order, numbered from 0), for the per-island residual stop; and each group's island count.
__global__ void k_row_island(uint32_t n, const uint32_t* __restrict__ rows, const uint32_t* __restrict__ run_flag,
                             const uint32_t* __restrict__ run_pre, uint32_t* row_isl) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) row_isl[rows[s]] = run_pre[s] + run_flag[s] - 1;
}
__global__ void k_local_isl_flags(uint32_t n, const uint32_t* __restrict__ ord, const uint32_t* __restrict__ gkey,
                                  const uint32_t* __restrict__ row_isl, uint32_t* flag) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  flag[p] = (p == 0 || gkey[p - 1] != gkey[p] || row_isl[ord[p - 1]] != row_isl[ord[p]]) ? 1u : 0u;
}
__global__ void k_local_isl(uint32_t n, const uint32_t* __restrict__ ord, const uint32_t* __restrict__ gkey,
                            const uint32_t* __restrict__ g_start, const uint32_t* __restrict__ g_cnt,
                            const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pre, uint32_t* row_lisl,
                            uint32_t* g_nisl) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  uint32_t g = gkey[p], s0 = g_start[g];
  uint32_t li = (pre[p] + flag[p]) - (pre[s0] + 1u);
  row_lisl[ord[p]] = li;
  if (p == s0 + g_cnt[g] - 1) g_nisl[g] = li + 1;
}
struct SRowsV {
  uint2* loc; uint32_t* flags; float2* inv; float4 *ra, *rb, *n, *t1, *t2, *mu, *va, *vb; float* jn; float2* jt; int* wm;
  float4* pred;  // learned warm start: (normal, friction 1, friction 2) in impulse units, w = 1 when valid
};
// Rows in schedule order, with local body indices and the constant velocity of a side that
// cannot move (a static or sleeping body's velocity at the contact; zero for terrain).
// Joint rows (index >= nc) carry no warm-cache index and no prediction; the fixed side of an angular
// joint row is that body's angular velocity.
__global__ void k_permute_rows(uint32_t n, uint32_t nc, const uint32_t* __restrict__ ord, RowsV R, BodiesV B,
                               const uint32_t* __restrict__ body_local, const int* __restrict__ wm_idx,
                               const uint32_t* __restrict__ row_lisl, const float* __restrict__ pred3,
                               const uint32_t* __restrict__ row_group, const uint32_t* __restrict__ g_class,
                               float4* pred_used, uint32_t cold_only, SRowsV O) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t r = ord[s];
  uint2 x = R.ab[r];
  uint32_t f = R.flags[r];
  float4 ra = R.ra[r], rb = R.rb[r];
  O.loc[s] = make_uint2((f & RF_TA) ? body_local[x.x] : 0xFFFFFFFFu, (f & RF_TB) ? body_local[x.y] : 0xFFFFFFFFu);
  O.flags[s] = (f & 0xFFFFu) | (row_lisl[r] << 16);  // bits 16..31: the row's island inside its group
  O.inv[s] = R.inv[r];
  O.ra[s] = ra; O.rb[s] = rb; O.n[s] = R.n[r]; O.t1[s] = R.t1[r]; O.t2[s] = R.t2[r]; O.mu[s] = R.mu[r];
  f3 va = mk3(0, 0, 0), vb = mk3(0, 0, 0);
  const bool jang = (f & RF_JANG) != 0;
  const bool jleg = (f & RF_JLEG) != 0;  // the original distance row reads linear velocities alone
  if (!(f & RF_TA))
    va = jang ? xyz(B.ang[x.x]) : (jleg ? xyz(B.lin[x.x]) : xyz(B.lin[x.x]) + cross(xyz(B.ang[x.x]), xyz(ra)));
  if (!(f & RF_TERRAIN) && !(f & RF_TB))
    vb = jang ? xyz(B.ang[x.y]) : (jleg ? xyz(B.lin[x.y]) : xyz(B.lin[x.y]) + cross(xyz(B.ang[x.y]), xyz(rb)));
  O.va[s] = f4(va);
  O.vb[s] = f4(vb);
  O.jn[s] = 0.0f;
  O.jt[s] = make_float2(0.0f, 0.0f);
  const bool contact = r < nc;
  O.wm[s] = contact ? wm_idx[r] : -1;
  // predictions reach every solver class except the global-memory one (islands beyond 4500 bodies)
  float4 p = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  // (cold_only: only rows the previous tick's cache has nothing for)
  if (contact && pred3 && g_class[row_group[r]] != 2u && (!cold_only || wm_idx[r] < 0))
    p = make_float4(pred3[3 * r], pred3[3 * r + 1], pred3[3 * r + 2], 1.0f);
  O.pred[s] = p;
  if (pred_used && contact) pred_used[r] = p;
}

// Shared-memory body state of one group
struct SBodies { float4* lin; float4* ang; float* Iw; float* im; };
// vfix: the velocity at the contact of the side that cannot move (a scheduled row has at most one)
struct SRow {
  uint32_t la, lb, flags;
  float inv_a, inv_b;
  f3 ra, rb, n, t1, t2, vfix;
  float m_n, m_t1, m_t2, mu_s, mu_k, sv, bias;
};
__device__ __forceinline__ SRow ld_srow(const SRowsV& R, uint32_t s) {
  SRow r;
  uint2 l = R.loc[s]; r.la = l.x; r.lb = l.y; r.flags = R.flags[s];
  float2 iv = R.inv[s]; r.inv_a = iv.x; r.inv_b = iv.y;
  float4 a = R.ra[s], b = R.rb[s], n = R.n[s], t1 = R.t1[s], t2 = R.t2[s], mu = R.mu[s];
  r.ra = xyz(a); r.m_n = a.w; r.rb = xyz(b); r.m_t1 = b.w; r.n = xyz(n); r.m_t2 = n.w;
  r.t1 = xyz(t1); r.bias = t1.w; r.t2 = xyz(t2);
  r.mu_s = mu.x; r.mu_k = mu.y; r.sv = mu.z;
  r.vfix = l.x == 0xFFFFFFFFu ? xyz(R.va[s]) : xyz(R.vb[s]);
  return r;
}
__device__ __forceinline__ f3 rel_vel_s(const SBodies& B, const SRow& r) {
  f3 va = r.la != 0xFFFFFFFFu ? xyz(B.lin[r.la]) + cross(xyz(B.ang[r.la]), r.ra) : r.vfix;
  f3 vb = (r.flags & RF_TERRAIN) ? mk3(0, 0, 0) : (r.lb != 0xFFFFFFFFu ? xyz(B.lin[r.lb]) + cross(xyz(B.ang[r.lb]), r.rb) : r.vfix);
  return vb - va;
}
__device__ __forceinline__ void body_impulse_s(const SBodies& B, uint32_t l, f3 j, f3 tau) {
  float im = B.im[l];
  if (im > 0.0f && vfin(j)) { float4 v = B.lin[l]; B.lin[l] = f4(fin_v(xyz(v) + j * im), v.w); }
  if (im > 0.0f && vfin(tau)) {
    const float* q = B.Iw + 9 * l;
    m3 Iw = mcols(mk3(q[0], q[1], q[2]), mk3(q[3], q[4], q[5]), mk3(q[6], q[7], q[8]));
    f3 dw = mvec(Iw, tau);
    float4 a = B.ang[l];
    B.ang[l] = f4(fin_v(xyz(a) + dw), a.w);
  }
}
__device__ __forceinline__ void contact_impulse_s(const SBodies& B, const SRow& r, f3 j) {
  if (r.inv_a > 0.0f) { f3 nj = -j; body_impulse_s(B, r.la, nj, cross(r.ra, nj)); }
  if (r.inv_b > 0.0f) body_impulse_s(B, r.lb, j, cross(r.rb, j));
}
__device__ __forceinline__ float mu_dynamic_s(const SRow& r, float slip) { return mu_law(r.mu_s, r.mu_k, r.sv, slip); }
__device__ __forceinline__ void warm_apply_s(const SBodies& B, const SRow& r, uint32_t s, float4 ea, float4 eb,
                                             float* jn_arr, float2* jt_arr) {
  float jn = ea.w;
  f3 jt = xyz(eb);
  jn_arr[s] = jn;
  f3 imp = r.n * jn;
  f3 v = rel_vel_s(B, r);
  float a = dot(v, r.t1), b = dot(v, r.t2);
  float mu = mu_dynamic_s(r, sqrtf(a * a + b * b));
  f3 t = clamp_length_max(mk3(dot(jt, r.t1), dot(jt, r.t2), 0.0f), mu * jn);
  jt_arr[s] = make_float2(t.x, t.y);
  imp = imp + ((r.t1 * t.x) + (r.t2 * t.y));
  contact_impulse_s(B, r, imp);
}
__device__ __forceinline__ float pgs_row_s(const SBodies& B, const SRow& r, uint32_t s, float* jn_arr, float2* jt_arr) {
  float v_rel_n = dot(rel_vel_s(B, r), r.n);
  float jn_raw = (r.bias - v_rel_n) * r.m_n;
  float old_jn = jn_arr[s];
  float new_jn = rmax(old_jn + jn_raw, 0.0f);
  jn_arr[s] = new_jn;
  contact_impulse_s(B, r, r.n * (new_jn - old_jn));
  f3 vf = rel_vel_s(B, r);
  float vt1 = dot(vf, r.t1), vt2 = dot(vf, r.t2);
  float slip = sqrtf(vt1 * vt1 + vt2 * vt2);
  float mu = mu_dynamic_s(r, slip);
  float2 ot = jt_arr[s];
  f3 old_t = mk3(ot.x, ot.y, 0.0f);
  f3 new_t = clamp_length_max(old_t - mk3(vt1 * r.m_t1, vt2 * r.m_t2, 0.0f), mu * new_jn);
  jt_arr[s] = make_float2(new_t.x, new_t.y);
  f3 d = new_t - old_t;
  contact_impulse_s(B, r, (r.t1 * d.x) + (r.t2 * d.y));
  float res = 0.0f;
  if (r.m_n > 0.0f) res = rmax(res, fabsf(new_jn - old_jn) / r.m_n);
  if (r.m_t1 > 0.0f) res = rmax(res, fabsf(d.x) / r.m_t1);
  if (r.m_t2 > 0.0f) res = rmax(res, fabsf(d.y) / r.m_t2);
  return res;
}
// pgs_row_s with the two bodies' velocities held in registers across the row (loaded once,
// written back once) and the residual's divisions left to the caller: the same operations in
// the same order, so the same bits, with a shorter dependent chain per level. dres receives
// new_jn - old_jn and the two friction deltas; the row's residual is
// max(|dres.x| / m_n, |dres.y| / m_t1, |dres.z| / m_t2) over the effective masses that are > 0.
__device__ __forceinline__ void impulse_reg(f3& lin, f3& ang, float im, const m3& Iw, f3 j, f3 tau) {
  if (im > 0.0f && vfin(j)) lin = fin_v(lin + j * im);
  if (im > 0.0f && vfin(tau)) ang = fin_v(ang + mvec(Iw, tau));
}
// impulse_reg on side `on` of a row, with its conditions as selects instead of branches: the new
// velocities are computed unconditionally and kept where impulse_reg would write them (the same
// expressions, so the same bits), so the two sides of a row interleave on one dependent chain
__device__ __forceinline__ f3 sel3(bool c, f3 a, f3 b) { return mk3(c ? a.x : b.x, c ? a.y : b.y, c ? a.z : b.z); }
__device__ __forceinline__ void impulse_sel(f3& lin, f3& ang, bool on, float im, const m3& Iw, f3 j, f3 tau) {
  const bool mv = on && im > 0.0f;
  const f3 nl = fin_v(lin + j * im), na = fin_v(ang + mvec(Iw, tau));
  lin = sel3(mv && vfin(j), nl, lin);
  ang = sel3(mv && vfin(tau), na, ang);
}
__device__ __forceinline__ m3 load_iw(const float* q) {
  return mcols(mk3(q[0], q[1], q[2]), mk3(q[3], q[4], q[5]), mk3(q[6], q[7], q[8]));
}
// ---- joint velocity rows (solver.rs:291-307 joint_row_vel / joint_row_apply, :821-830 the update):
// v = (v_b - v_a) . u over the anchors (linear) or the angular velocities (angular); the impulse
// stays in [lam_min, lam_max] = (mu_s, mu_k) of the row; bias is the target, m_n = 1 / k.
__device__ __forceinline__ void joint_apply_reg(f3& la, f3& aa, f3& lb, f3& ab, const SRow& r, const m3& qa, const m3& qb,
                                                float ima, float imb, float lam) {
  f3 p = r.n * lam;
  const bool ia = r.inv_a > 0.0f, ib = r.inv_b > 0.0f;
  const f3 np = -p;
  if (r.flags & RF_JANG) {  // selects, as impulse_sel
    const f3 na = fin_v(aa + mvec(qa, np)), nb = fin_v(ab + mvec(qb, p));
    aa = sel3(ia && ima > 0.0f && vfin(np), na, aa);
    ab = sel3(ib && imb > 0.0f && vfin(p), nb, ab);
  } else {
    impulse_sel(la, aa, ia, ima, qa, np, cross(r.ra, np));
    impulse_sel(lb, ab, ib, imb, qb, p, cross(r.rb, p));
  }
}
// The original distance row (solver.rs:793-817) on register copies of the two linear velocities
// (a side outside the group reads vfix, its linear velocity): returns the impulse.
__device__ __forceinline__ float legacy_row_reg(f3& la, f3& lb, bool ha, bool hb, const SRow& r, float ima, float imb) {
  float v_rel = dot((hb ? lb : r.vfix) - (ha ? la : r.vfix), r.n);
  float j_mag = -(v_rel + r.bias) / r.m_t1;
  f3 pa = (-r.n) * j_mag, pb = r.n * j_mag;
  if (r.inv_a > 0.0f && ima > 0.0f && vfin(pa)) la = fin_v(la + pa * ima);
  if (r.inv_b > 0.0f && imb > 0.0f && vfin(pb)) lb = fin_v(lb + pb * imb);
  return j_mag;
}
__device__ __noinline__ void joint_row_core(float4* lin, float4* ang, const SRow& r, const m3& qa, const m3& qb,
                                               float ima, float imb, float& acc, float* d3) {
  const bool ha = r.la != 0xFFFFFFFFu, hb = r.lb != 0xFFFFFFFFu;
  const bool ia = r.inv_a > 0.0f, ib = r.inv_b > 0.0f;
  float4 LA = make_float4(0, 0, 0, 0), AA = LA, LB = LA, AB = LA;
  if (ha) { LA = lin[r.la]; AA = ang[r.la]; }
  if (hb) { LB = lin[r.lb]; AB = ang[r.lb]; }
  f3 la = xyz(LA), aa = xyz(AA), lb = xyz(LB), ab = xyz(AB);
  if (r.flags & RF_JNULL) {
    d3[0] = 0.0f;
    d3[1] = 0.0f;
    d3[2] = 0.0f;
    return;
  }
  if (r.flags & RF_JLEG) {
    d3[0] = legacy_row_reg(la, lb, ha, hb, r, ima, imb);
    d3[1] = 0.0f;
    d3[2] = 0.0f;
    if (ia) lin[r.la] = f4(la, LA.w);
    if (ib) lin[r.lb] = f4(lb, LB.w);
    return;
  }
  f3 va, vb;
  if (r.flags & RF_JANG) { va = ha ? aa : r.vfix; vb = hb ? ab : r.vfix; }
  else { va = ha ? la + cross(aa, r.ra) : r.vfix; vb = hb ? lb + cross(ab, r.rb) : r.vfix; }
  float v = dot(vb - va, r.n);
  float old = acc;
  float nw = clampf(joint_lam(old, r.bias, v, r.t1.z, r.m_n), r.mu_s, r.mu_k);
  acc = nw;
  if (nw != old) {
    joint_apply_reg(la, aa, lb, ab, r, qa, qb, ima, imb, nw - old);
    if (ia) { lin[r.la] = f4(la, LA.w); ang[r.la] = f4(aa, AA.w); }
    if (ib) { lin[r.lb] = f4(lb, LB.w); ang[r.lb] = f4(ab, AB.w); }
  }
  d3[0] = nw - old;
  d3[1] = 0.0f;
  d3[2] = 0.0f;
}
// A joint unit on shared-memory bodies: the joint's rows in order, with both bodies' velocities,
// inverse inertias and inverse masses held in registers across them (every row of a joint moves the
// same two bodies) -- the same operations in the same order as one joint_row_core per row.
__device__ __noinline__ void joint_unit_core(float4* lin, float4* ang, const SRow* rows, uint32_t cnt, const float* Iw,
                                             const float* im, float* jn, float* dres) {
  const SRow& r0 = rows[0];
  const bool ha = r0.la != 0xFFFFFFFFu, hb = r0.lb != 0xFFFFFFFFu;
  const bool ia = r0.inv_a > 0.0f, ib = r0.inv_b > 0.0f;
  const m3 qa = load_iw(ia ? Iw + 9 * (size_t)r0.la : Iw), qb = load_iw(ib ? Iw + 9 * (size_t)r0.lb : Iw);
  const float ima = ia ? im[r0.la] : 0.0f, imb = ib ? im[r0.lb] : 0.0f;
  float4 LA = make_float4(0, 0, 0, 0), AA = LA, LB = LA, AB = LA;
  if (ha) { LA = lin[r0.la]; AA = ang[r0.la]; }
  if (hb) { LB = lin[r0.lb]; AB = ang[r0.lb]; }
  f3 la = xyz(LA), aa = xyz(AA), lb = xyz(LB), ab = xyz(AB);
  bool moved = false;
  for (uint32_t q = 0; q < cnt; ++q) {
    const SRow& r = rows[q];
    if (r.flags & RF_JNULL) {
      dres[3 * q] = 0.0f;
      dres[3 * q + 1] = 0.0f;
      dres[3 * q + 2] = 0.0f;
      continue;
    }
    if (r.flags & RF_JLEG) {
      dres[3 * q] = legacy_row_reg(la, lb, ha, hb, r, ima, imb);
      dres[3 * q + 1] = 0.0f;
      dres[3 * q + 2] = 0.0f;
      moved = true;
      continue;
    }
    f3 va, vb;
    if (r.flags & RF_JANG) { va = ha ? aa : r.vfix; vb = hb ? ab : r.vfix; }
    else { va = ha ? la + cross(aa, r.ra) : r.vfix; vb = hb ? lb + cross(ab, r.rb) : r.vfix; }
    float v = dot(vb - va, r.n);
    float old = jn[q];
    float nw = clampf(joint_lam(old, r.bias, v, r.t1.z, r.m_n), r.mu_s, r.mu_k);
    jn[q] = nw;
    if (nw != old) {
      joint_apply_reg(la, aa, lb, ab, r, qa, qb, ima, imb, nw - old);
      moved = true;
    }
    dres[3 * q] = nw - old;
    dres[3 * q + 1] = 0.0f;
    dres[3 * q + 2] = 0.0f;
  }
  if (moved) {
    if (ia) { lin[r0.la] = f4(la, LA.w); ang[r0.la] = f4(aa, AA.w); }
    if (ib) { lin[r0.lb] = f4(lb, LB.w); ang[r0.lb] = f4(ab, AB.w); }
  }
}
// The row update on bodies whose velocities live in lin / ang (shared memory), with both bodies'
// world inverse inertia and inverse mass passed in; jn / jt are the row's accumulators, d3
// receives (new_jn - old_jn, friction deltas) for the residual.
__device__ __forceinline__ void pgs_row_core(float4* lin, float4* ang, const SRow& r, const m3& qa, const m3& qb,
                                             float ima, float imb, float& jn_acc, float2& jt_acc, float* d3) {
  if (r.flags & RF_JOINT) { joint_row_core(lin, ang, r, qa, qb, ima, imb, jn_acc, d3); return; }
  const bool ha = r.la != 0xFFFFFFFFu, hb = !(r.flags & RF_TERRAIN) && r.lb != 0xFFFFFFFFu;
  const bool ia = r.inv_a > 0.0f, ib = r.inv_b > 0.0f;
  float4 LA = make_float4(0, 0, 0, 0), AA = LA, LB = LA, AB = LA;
  if (ha || ia) { LA = lin[r.la]; AA = ang[r.la]; }
  if (hb || ib) { LB = lin[r.lb]; AB = ang[r.lb]; }
  f3 la = xyz(LA), aa = xyz(AA), lb = xyz(LB), ab = xyz(AB);
  auto rel = [&]() {
    f3 va = ha ? la + cross(aa, r.ra) : r.vfix;
    f3 vb = (r.flags & RF_TERRAIN) ? mk3(0, 0, 0) : (hb ? lb + cross(ab, r.rb) : r.vfix);
    return vb - va;
  };
  auto apply = [&](f3 j) {
    const f3 nj = -j;
    impulse_sel(la, aa, ia, ima, qa, nj, cross(r.ra, nj));
    impulse_sel(lb, ab, ib, imb, qb, j, cross(r.rb, j));
  };
  float v_rel_n = dot(rel(), r.n);
  float jn_raw = (r.bias - v_rel_n) * r.m_n;
  float old_jn = jn_acc;
  float new_jn = rmax(old_jn + jn_raw, 0.0f);
  jn_acc = new_jn;
  apply(r.n * (new_jn - old_jn));
  f3 vf = rel();
  float vt1 = dot(vf, r.t1), vt2 = dot(vf, r.t2);
  float slip = sqrtf(vt1 * vt1 + vt2 * vt2);
  float mu = mu_dynamic_s(r, slip);
  float2 ot = jt_acc;
  f3 old_t = mk3(ot.x, ot.y, 0.0f);
  f3 new_t = clamp_length_max(old_t - mk3(vt1 * r.m_t1, vt2 * r.m_t2, 0.0f), mu * new_jn);
  jt_acc = make_float2(new_t.x, new_t.y);
  f3 d = new_t - old_t;
  apply((r.t1 * d.x) + (r.t2 * d.y));
  if (ia) { lin[r.la] = f4(la, LA.w); ang[r.la] = f4(aa, AA.w); }
  if (ib) { lin[r.lb] = f4(lb, LB.w); ang[r.lb] = f4(ab, AB.w); }
  d3[0] = new_jn - old_jn;
  d3[1] = d.x;
  d3[2] = d.y;
}
// warm_apply_s on register copies (same operations, same order)
__device__ __forceinline__ void warm_core(float4* lin, float4* ang, const SRow& r, const m3& qa, const m3& qb,
                                          float ima, float imb, float4 ea, float4 eb, float& jn_acc, float2& jt_acc) {
  const bool ha = r.la != 0xFFFFFFFFu, hb = !(r.flags & RF_TERRAIN) && r.lb != 0xFFFFFFFFu;
  const bool ia = r.inv_a > 0.0f, ib = r.inv_b > 0.0f;
  float4 LA = make_float4(0, 0, 0, 0), AA = LA, LB = LA, AB = LA;
  if (ha || ia) { LA = lin[r.la]; AA = ang[r.la]; }
  if (hb || ib) { LB = lin[r.lb]; AB = ang[r.lb]; }
  f3 la = xyz(LA), aa = xyz(AA), lb = xyz(LB), ab = xyz(AB);
  float jn = ea.w;
  f3 jt = xyz(eb);
  jn_acc = jn;
  f3 imp = r.n * jn;
  f3 va = ha ? la + cross(aa, r.ra) : r.vfix;
  f3 vb = (r.flags & RF_TERRAIN) ? mk3(0, 0, 0) : (hb ? lb + cross(ab, r.rb) : r.vfix);
  f3 v = vb - va;
  float a = dot(v, r.t1), b = dot(v, r.t2);
  float mu = mu_dynamic_s(r, sqrtf(a * a + b * b));
  f3 t = clamp_length_max(mk3(dot(jt, r.t1), dot(jt, r.t2), 0.0f), mu * jn);
  jt_acc = make_float2(t.x, t.y);
  imp = imp + ((r.t1 * t.x) + (r.t2 * t.y));
  const f3 nimp = -imp;
  impulse_sel(la, aa, ia, ima, qa, nimp, cross(r.ra, nimp));
  impulse_sel(lb, ab, ib, imb, qb, imp, cross(r.rb, imp));
  if (ia) { lin[r.la] = f4(la, LA.w); ang[r.la] = f4(aa, AA.w); }
  if (ib) { lin[r.lb] = f4(lb, LB.w); ang[r.lb] = f4(ab, AB.w); }
}
// Learned warm start: the row's normal velocity error |bias - v_rel . n| after a candidate start
// (applied to register copies, nothing written), and the choice between the previous tick's
// impulse (or none) and the predicted one: the prediction is kept only when it leaves the smaller
// error. Returns 1 when the prediction was applied.
__device__ __forceinline__ float warm_trial_err(const float4* lin, const float4* ang, const SRow& r, const m3& qa,
                                                const m3& qb, float ima, float imb, bool apply_start, float4 ea, float4 eb) {
  const bool ha = r.la != 0xFFFFFFFFu, hb = !(r.flags & RF_TERRAIN) && r.lb != 0xFFFFFFFFu;
  const bool ia = r.inv_a > 0.0f, ib = r.inv_b > 0.0f;
  f3 la = mk3(0, 0, 0), aa = la, lb = la, ab = la;
  if (ha || ia) { la = xyz(lin[r.la]); aa = xyz(ang[r.la]); }
  if (hb || ib) { lb = xyz(lin[r.lb]); ab = xyz(ang[r.lb]); }
  auto rel = [&]() {
    f3 va = ha ? la + cross(aa, r.ra) : r.vfix;
    f3 vb = (r.flags & RF_TERRAIN) ? mk3(0, 0, 0) : (hb ? lb + cross(ab, r.rb) : r.vfix);
    return vb - va;
  };
  if (apply_start) {
    float jn = ea.w;
    f3 jt = xyz(eb);
    f3 imp = r.n * jn;
    f3 v = rel();
    float a = dot(v, r.t1), b = dot(v, r.t2);
    float mu = mu_dynamic_s(r, sqrtf(a * a + b * b));
    f3 t = clamp_length_max(mk3(dot(jt, r.t1), dot(jt, r.t2), 0.0f), mu * jn);
    imp = imp + ((r.t1 * t.x) + (r.t2 * t.y));
    if (ia) { f3 nj = -imp; impulse_reg(la, aa, ima, qa, nj, cross(r.ra, nj)); }
    if (ib) impulse_reg(lb, ab, imb, qb, imp, cross(r.rb, imp));
  }
  return fabsf(r.bias - dot(rel(), r.n));
}
__device__ __forceinline__ int warm_select(float4* lin, float4* ang, const SRow& r, const m3& qa, const m3& qb, float ima,
                                           float imb, bool has_ref, float4 ea, float4 eb, float4 pred, float& jn_acc,
                                           float2& jt_acc) {
  if (r.flags & RF_JOINT) {  // impulse applied by k_joint_warm before every contact's warm start
    jn_acc = (r.flags & RF_JWARM) ? r.t2.x : 0.0f;
    return 0;
  }
  if (pred.w == 0.0f) {
    if (has_ref) warm_core(lin, ang, r, qa, qb, ima, imb, ea, eb, jn_acc, jt_acc);
    return 0;
  }
  const float su = r.m_n * kImpulseUnit;
  float4 pa = make_float4(0.0f, 0.0f, 0.0f, rmax(pred.x * su, 0.0f));
  float4 pb = f4((r.t1 * (pred.y * su)) + (r.t2 * (pred.z * su)));
  float e_ref = warm_trial_err(lin, ang, r, qa, qb, ima, imb, has_ref, ea, eb);
  float e_pred = warm_trial_err(lin, ang, r, qa, qb, ima, imb, true, pa, pb);
  if (e_pred < e_ref) {
    warm_core(lin, ang, r, qa, qb, ima, imb, pa, pb, jn_acc, jt_acc);
    return 1;
  }
  if (has_ref) warm_core(lin, ang, r, qa, qb, ima, imb, ea, eb, jn_acc, jt_acc);
  return 0;
}
__device__ __forceinline__ void pgs_row_reg(const SBodies& B, const SRow& r, uint32_t s, float* jn_arr, float2* jt_arr,
                                            float* dres) {
  const bool ia = r.inv_a > 0.0f, ib = r.inv_b > 0.0f;
  const m3 qa = load_iw(ia ? B.Iw + 9 * (size_t)r.la : B.Iw);  // loaded once for both impulses
  const m3 qb = load_iw(ib ? B.Iw + 9 * (size_t)r.lb : B.Iw);
  float ima = ia ? B.im[r.la] : 0.0f, imb = ib ? B.im[r.lb] : 0.0f;
  pgs_row_core(B.lin, B.ang, r, qa, qb, ima, imb, jn_arr[s], jt_arr[s], dres + 3 * (size_t)s);
}
__device__ __forceinline__ float row_residual(const SRow& r, const float* dres, uint32_t s) {
  float res = 0.0f;
  if (r.m_n > 0.0f) res = rmax(res, fabsf(dres[3 * s]) / r.m_n);
  if (r.m_t1 > 0.0f) res = rmax(res, fabsf(dres[3 * s + 1]) / r.m_t1);
  if (r.m_t2 > 0.0f) res = rmax(res, fabsf(dres[3 * s + 2]) / r.m_t2);
  return res;
}

// Per-island residual stop, shared by the group kernels below: after each sweep an island whose
// rows changed no velocity by more than tol is done and its rows are skipped from then on
// (islands share no body, so the other islands' arithmetic is unchanged). Fixed-iteration mode
// (tol = 0) never marks an island done.

// A group solved by one block with everything it touches in that block's shared memory: rows
// (in schedule order), impulses, bodies, level starts and per-island residual state; a block
// barrier between levels. Same arithmetic and order as the serial sweep. Capacities RC rows,
// BC bodies, IC islands set the layout: packed groups (class 3) 64 / 128 / 64 in about 20 KB
// with 64 threads; single islands (classes 10..15) R / R + 1 / 1 for R = 128 ... 1024 rows,
// about 220 bytes per row (28 KB ... 225 KB), with 128 threads.
struct OnchipLayout {
  uint32_t RC, BC, IC;
  uint32_t o_lin, o_ang, o_jt, o_rows, o_jn, o_dres, o_Iw, o_im, o_lvl, o_res, o_last, o_sw, o_done, bytes;
};
__host__ __device__ inline uint32_t onchip_take(uint32_t& o, uint32_t bytes) {
  uint32_t a = o;
  o = (o + bytes + 15u) & ~15u;
  return a;
}
__host__ __device__ inline OnchipLayout onchip_layout(uint32_t RC, uint32_t BC, uint32_t IC) {
  OnchipLayout L;
  L.RC = RC; L.BC = BC; L.IC = IC;
  uint32_t o = 0;
  L.o_lin = onchip_take(o, 16u * BC);
  L.o_ang = onchip_take(o, 16u * BC);
  L.o_jt = onchip_take(o, 8u * RC);
  L.o_rows = onchip_take(o, (uint32_t)sizeof(SRow) * RC);
  L.o_jn = onchip_take(o, 4u * RC);
  L.o_dres = onchip_take(o, 12u * RC);
  L.o_Iw = onchip_take(o, 36u * BC);
  L.o_im = onchip_take(o, 4u * BC);
  L.o_lvl = onchip_take(o, 4u * (RC + 1u));
  L.o_res = onchip_take(o, 4u * IC);
  L.o_last = onchip_take(o, 4u * IC);
  L.o_sw = onchip_take(o, 4u * IC);
  L.o_done = onchip_take(o, IC);
  L.bytes = o;
  return L;
}
// threads of a packed-group block (32, 64 or 128) and of a single-island block (32 to 256) are
// tuning knobs (WorldGpu::Tuning); each value has its own instantiation below
template <bool MULTI, int NT>
__global__ void __launch_bounds__(NT) k_vel_solve_onchip(OnchipLayout Lo, uint32_t g0, uint32_t ng,
                                                         const uint32_t* __restrict__ glist, uint32_t want_class,
                                                         const uint32_t* __restrict__ g_class,
                                                         const uint32_t* __restrict__ gb_start,
                                                         const uint32_t* __restrict__ gb_cnt,
                                                         const uint32_t* __restrict__ gb_list,
                                                         const uint32_t* __restrict__ g_nisl, Sched S, SRowsV R,
                                                         BodiesV G, const float4* __restrict__ wa,
                                                         const float4* __restrict__ wb, float* acc_jn, float2* acc_jt,
                                                         int iters, float tol, uint32_t* stats,
                                                         const uint32_t* __restrict__ row_islid, uint32_t* isl_final) {
  if (glist && blockIdx.x >= ng) return;
  uint32_t g = glist ? glist[blockIdx.x] : g0 + blockIdx.x;
  if (!glist && g >= ng) return;
  if (g_class[g] != want_class) return;
  extern __shared__ float4 wsm_raw[];
  unsigned char* sb = reinterpret_cast<unsigned char*>(wsm_raw);
  struct {
    float4 *lin, *ang; float2* jt; SRow* rows; float *jn, *dres, *Iw, *im;
    uint32_t *lvl, *isl_res, *isl_last, *isl_sw; uint8_t* isl_done;
  } W{reinterpret_cast<float4*>(sb + Lo.o_lin), reinterpret_cast<float4*>(sb + Lo.o_ang),
      reinterpret_cast<float2*>(sb + Lo.o_jt), reinterpret_cast<SRow*>(sb + Lo.o_rows),
      reinterpret_cast<float*>(sb + Lo.o_jn), reinterpret_cast<float*>(sb + Lo.o_dres),
      reinterpret_cast<float*>(sb + Lo.o_Iw), reinterpret_cast<float*>(sb + Lo.o_im),
      reinterpret_cast<uint32_t*>(sb + Lo.o_lvl), reinterpret_cast<uint32_t*>(sb + Lo.o_res),
      reinterpret_cast<uint32_t*>(sb + Lo.o_last), reinterpret_cast<uint32_t*>(sb + Lo.o_sw), sb + Lo.o_done};
  const uint32_t RC = Lo.RC, BC = Lo.BC, IC = Lo.IC;
  __shared__ uint32_t red[NT / 32][4];
  const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const uint32_t nbg = gb_cnt[g], b0 = gb_start[g], nisl = g_nisl[g];
  const uint32_t off = S.lvl_off[g], nl = S.nlev[g];
  const uint32_t base = S.lvl_start[off], nr = S.lvl_start[off + nl] - base;
  if (nbg > BC || nr > RC || nisl > IC) {  // not reached: the class was chosen by these sizes
    if (tid == 0) atomicOr(&stats[STAT_ERR], 2u);
    return;
  }
  for (uint32_t i = tid; i < nbg; i += NT) {
    uint32_t b = gb_list[b0 + i];
    W.lin[i] = G.lin[b];
    W.ang[i] = G.ang[b];
    for (int k = 0; k < 9; ++k) W.Iw[9 * i + k] = G.Iw[9 * (size_t)b + k];
    W.im[i] = G.inv_mass[b];
  }
  for (uint32_t i = tid; i < nr; i += NT) {
    W.rows[i] = ld_srow(R, base + i);
    W.jn[i] = 0.0f;
    W.jt[i] = make_float2(0.0f, 0.0f);
  }
  for (uint32_t L = tid; L <= nl; L += NT) W.lvl[L] = S.lvl_start[off + L] - base;
  for (uint32_t i = tid; i < nisl; i += NT) { W.isl_res[i] = 0u; W.isl_last[i] = 0u; W.isl_sw[i] = 0u; W.isl_done[i] = 0; }
  __syncthreads();
  SBodies B{W.lin, W.ang, W.Iw, W.im};
  // Between two levels of at most 32 rows only the first warp works and a warp barrier orders its
  // shared-memory writes; a block barrier is taken only where a wider level begins or ends (every
  // warp takes the same barriers: the condition depends on the level sizes alone).
  auto wide = [&](uint32_t L) { return L < nl && W.lvl[L + 1] - W.lvl[L] > 32u; };
  auto level_sync = [&](uint32_t L) {
    if (NT == 32 || wide(L) || wide(L + 1)) __syncthreads();
    else __syncwarp();
  };
  uint32_t n_pred = 0;
  for (uint32_t L = 0; L < nl; ++L) {
    for (uint32_t i = W.lvl[L] + tid; i < W.lvl[L + 1] && (wid == 0 || wide(L)); i += NT) {
      int e = R.wm[base + i];
      float4 p = R.pred[base + i];
      const SRow& r = W.rows[i];
      if (e < 0 && p.w == 0.0f && !(r.flags & RF_JWARM)) continue;
      const bool ia = r.inv_a > 0.0f, ib = r.inv_b > 0.0f;
      const m3 qa = load_iw(ia ? B.Iw + 9 * (size_t)r.la : B.Iw), qb = load_iw(ib ? B.Iw + 9 * (size_t)r.lb : B.Iw);
      n_pred += warm_select(B.lin, B.ang, r, qa, qb, ia ? B.im[r.la] : 0.0f, ib ? B.im[r.lb] : 0.0f, e >= 0,
                            e >= 0 ? wa[e] : make_float4(0, 0, 0, 0), e >= 0 ? wb[e] : make_float4(0, 0, 0, 0), p,
                            W.jn[i], W.jt[i]);
    }
    level_sync(L);
  }
  __syncthreads();
  if (n_pred) atomicAdd(&stats[STAT_PRED_USED], n_pred);
  int it = 0;
  while (it < iters) {
    for (uint32_t L = 0; L < nl; ++L) {
      for (uint32_t i = W.lvl[L] + tid; i < W.lvl[L + 1] && (wid == 0 || wide(L)); i += NT) {
        const SRow& r = W.rows[i];
        if (MULTI && W.isl_done[r.flags >> 16]) continue;
        if (r.flags & RF_JOINT) {  // a joint is one unit: its first row runs all its rows in order
          if (!(r.flags & RF_JFIRST)) continue;
          joint_unit_core(B.lin, B.ang, &W.rows[i], (uint32_t)r.t1.x, B.Iw, B.im, &W.jn[i], &W.dres[3 * (size_t)i]);
          continue;
        }
        pgs_row_reg(B, r, i, W.jn, W.jt, W.dres);
      }
      level_sync(L);
    }
    __syncthreads();
    // the sweep's residual per island, off the level chain (non-negative floats: integer max)
    if (!MULTI) {
      uint32_t m = 0;
      for (uint32_t i = tid; i < nr; i += NT) m = max(m, fbits(row_residual(W.rows[i], W.dres, i)));
      m = __reduce_max_sync(0xffffffffu, m);
      if (lane == 0) red[wid][0] = m;
      __syncthreads();
      if (tid == 0) {
        uint32_t x = 0;
        for (int w = 0; w < NT / 32; ++w) x = max(x, red[w][0]);
        W.isl_res[0] = x;
      }
    } else {
      for (uint32_t i = tid; i < nr; i += NT) {
        uint32_t li = W.rows[i].flags >> 16;
        if (!W.isl_done[li]) atomicMax(&W.isl_res[li], fbits(row_residual(W.rows[i], W.dres, i)));
      }
    }
    __syncthreads();
    it++;
    bool active = false;
    for (uint32_t i = tid; i < nisl; i += NT) {
      if (W.isl_done[i]) continue;
      uint32_t rb = W.isl_res[i];
      W.isl_res[i] = 0u;
      W.isl_sw[i] = (uint32_t)it;
      W.isl_last[i] = rb;
      if (tol > 0.0f && __uint_as_float(rb) <= tol) W.isl_done[i] = 1;
      else active = true;
    }
    if (!__syncthreads_or(active)) break;
  }
  for (uint32_t i = tid; i < nbg; i += NT) {
    uint32_t b = gb_list[b0 + i];
    G.lin[b] = W.lin[i];
    G.ang[b] = W.ang[i];
  }
  uint32_t my_rs = 0, my_rcap = 0;
  for (uint32_t i = tid; i < nr; i += NT) {
    uint32_t r = S.ord[base + i];
    acc_jn[r] = W.jn[i];
    acc_jt[r] = W.jt[i];
    const uint32_t li = MULTI ? W.rows[i].flags >> 16 : 0u;
    my_rs += W.isl_sw[li];
    if (tol > 0.0f && !W.isl_done[li]) my_rcap++;
    isl_final[row_islid[r]] = W.isl_last[li];  // every row of an island writes the same value
  }
  uint32_t my_sw = 0, my_res = 0, my_cap = 0;
  for (uint32_t i = tid; i < nisl; i += NT) {
    my_sw = max(my_sw, W.isl_sw[i]);
    my_res = max(my_res, W.isl_last[i]);
    if (tol > 0.0f && !W.isl_done[i]) my_cap++;
  }
  {
    const uint32_t rc = __reduce_add_sync(0xffffffffu, my_rcap);
    if (lane == 0 && rc) atomicAdd(&stats[STAT_ROWS_CAPPED], rc);
  }
  my_rs = __reduce_add_sync(0xffffffffu, my_rs);
  my_cap = __reduce_add_sync(0xffffffffu, my_cap);
  my_sw = __reduce_max_sync(0xffffffffu, my_sw);
  my_res = __reduce_max_sync(0xffffffffu, my_res);
  __syncthreads();
  if (lane == 0) { red[wid][0] = my_rs; red[wid][1] = my_cap; red[wid][2] = my_sw; red[wid][3] = my_res; }
  __syncthreads();
  if (tid == 0) {
    uint32_t a = 0, c = 0, w_ = 0, r_ = 0;
    for (int w = 0; w < NT / 32; ++w) { a += red[w][0]; c += red[w][1]; w_ = max(w_, red[w][2]); r_ = max(r_, red[w][3]); }
    if (a) atomicAdd(&stats[STAT_ROWSWEEPS], a);
    if (c) atomicAdd(&stats[STAT_ISLANDS_CAPPED], c);
    if (w_) atomicMax(&stats[STAT_SWEEPS], w_);
    if (r_) atomicMax(&stats[STAT_RESID], r_);
  }
}

// ------------------------------------------------------------------ big islands
// An island beyond the on-chip buckets (bodies and levels within its bucket's caps) solved by one
// CTA: body velocities in shared memory, rows streamed through a double-buffered stage. Each level
// is cut into chunks of at most CH rows (one per thread); while a chunk is solved, cp.async
// copies the next chunk -- its row data, both bodies' world inverse inertia and inverse mass
// (BigRowX, built per tick) and its accumulators -- into the other buffer, so the level chain
// never waits on L2. Accumulators (jn, jt) live in global memory between sweeps (BigJ).
template <int CH>
struct BigStage {
  float4 ra[CH], rb[CH], n[CH], t1[CH], t2[CH], mu[CH];
  float4 x[CH][7];  // Iw a (9) im a | Iw b (9) im b (3 float4 each: 12 floats), vfix
  float4 j[CH];     // jn, jt.x, jt.y
  uint2 loc[CH];
  float2 inv[CH];
  uint32_t flags[CH];
};
static_assert(sizeof(BigStage<64>) % 16 == 0 && sizeof(BigStage<128>) % 16 == 0, "stage buffers stay 16-byte aligned");
template <int CH>
constexpr size_t big_smem(uint32_t bodies, uint32_t levels) {
  return 2 * sizeof(BigStage<CH>) + 32u * (size_t)bodies + ((4u * (levels + 1u) + 15u) & ~15u);
}
static_assert(big_smem<128>(4500u, 4096u) + 16 <= 232448, "largest big-island block exceeds the shared memory limit");
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
// Per row (schedule position) of a big island: Iw and inverse mass of both bodies, vfix.
__global__ void k_big_rows_x(uint32_t n, const uint32_t* __restrict__ ord, const uint32_t* __restrict__ row_group,
                             const uint32_t* __restrict__ g_class, RowsV R, BodiesV B, SRowsV SR, float4* X, float4* J) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t r = ord[s];
  uint32_t c = g_class[row_group[r]];
  if (c < 20u || c >= 20u + BIG_BUCKETS) return;
  uint2 ab = R.ab[r];
  uint32_t f = R.flags[r];
  float q[24];
  for (int k = 0; k < 24; ++k) q[k] = 0.0f;
  if (f & RF_WA) { for (int k = 0; k < 9; ++k) q[k] = B.Iw[9 * (size_t)ab.x + k]; q[9] = B.inv_mass[ab.x]; }
  if (f & RF_WB) { for (int k = 0; k < 9; ++k) q[12 + k] = B.Iw[9 * (size_t)ab.y + k]; q[21] = B.inv_mass[ab.y]; }
  float4* o = X + 7 * (size_t)s;
  for (int k = 0; k < 6; ++k) o[k] = make_float4(q[4 * k], q[4 * k + 1], q[4 * k + 2], q[4 * k + 3]);
  uint2 l = SR.loc[s];
  o[6] = l.x == 0xFFFFFFFFu ? SR.va[s] : SR.vb[s];
  J[s] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}
template <int CH>
__device__ __forceinline__ void big_stage_issue(BigStage<CH>& st, uint32_t s0, uint32_t n, const SRowsV& R,
                                                const float4* __restrict__ X, const float4* J) {
  for (uint32_t i = threadIdx.x; i < n; i += CH) {
    uint32_t s = s0 + i;
    cp_async16(&st.ra[i], &R.ra[s]); cp_async16(&st.rb[i], &R.rb[s]); cp_async16(&st.n[i], &R.n[s]);
    cp_async16(&st.t1[i], &R.t1[s]); cp_async16(&st.t2[i], &R.t2[s]); cp_async16(&st.mu[i], &R.mu[s]);
    for (int k = 0; k < 7; ++k) cp_async16(&st.x[i][k], &X[7 * (size_t)s + k]);
    cp_async16(&st.j[i], &J[s]);
    cp_async8(&st.loc[i], &R.loc[s]); cp_async8(&st.inv[i], &R.inv[s]); cp_async4(&st.flags[i], &R.flags[s]);
  }
}
template <int CH>
__device__ __forceinline__ SRow big_row(const BigStage<CH>& st, uint32_t i, m3* qa, m3* qb, float* ima, float* imb) {
  SRow r;
  uint2 l = st.loc[i]; r.la = l.x; r.lb = l.y; r.flags = st.flags[i];
  float2 iv = st.inv[i]; r.inv_a = iv.x; r.inv_b = iv.y;
  float4 a = st.ra[i], b = st.rb[i], n = st.n[i], t1 = st.t1[i], t2 = st.t2[i], mu = st.mu[i];
  r.ra = xyz(a); r.m_n = a.w; r.rb = xyz(b); r.m_t1 = b.w; r.n = xyz(n); r.m_t2 = n.w;
  r.t1 = xyz(t1); r.bias = t1.w; r.t2 = xyz(t2);
  r.mu_s = mu.x; r.mu_k = mu.y; r.sv = mu.z;
  r.vfix = xyz(st.x[i][6]);
  float q[24];
  for (int k = 0; k < 6; ++k) { float4 v = st.x[i][k]; q[4 * k] = v.x; q[4 * k + 1] = v.y; q[4 * k + 2] = v.z; q[4 * k + 3] = v.w; }
  *qa = mcols(mk3(q[0], q[1], q[2]), mk3(q[3], q[4], q[5]), mk3(q[6], q[7], q[8]));
  *ima = q[9];
  *qb = mcols(mk3(q[12], q[13], q[14]), mk3(q[15], q[16], q[17]), mk3(q[18], q[19], q[20]));
  *imb = q[21];
  return r;
}
// A row of the big-island stream read straight from global memory (a joint unit's later rows, which
// may lie past the staged chunk).
__device__ __forceinline__ SRow big_row_global(const SRowsV& R, const float4* __restrict__ X, uint32_t s, m3* qa, m3* qb,
                                               float* ima, float* imb) {
  SRow r = ld_srow(R, s);
  const float4* x = X + 7 * (size_t)s;
  float q[24];
  for (int k = 0; k < 6; ++k) { float4 v = x[k]; q[4 * k] = v.x; q[4 * k + 1] = v.y; q[4 * k + 2] = v.z; q[4 * k + 3] = v.w; }
  *qa = mcols(mk3(q[0], q[1], q[2]), mk3(q[3], q[4], q[5]), mk3(q[6], q[7], q[8]));
  *ima = q[9];
  *qb = mcols(mk3(q[12], q[13], q[14]), mk3(q[15], q[16], q[17]), mk3(q[18], q[19], q[20]));
  *imb = q[21];
  return r;
}
template <int CH>
__global__ void __launch_bounds__(CH) k_vel_solve_big(uint32_t BC, uint32_t LC, uint32_t want_class,
                                                      uint32_t n_listed, const uint32_t* __restrict__ glist,
                                                           const uint32_t* __restrict__ g_class,
                                                           const uint32_t* __restrict__ gb_start,
                                                           const uint32_t* __restrict__ gb_cnt,
                                                           const uint32_t* __restrict__ gb_list, Sched S, SRowsV R,
                                                           const float4* __restrict__ X, float4* J, BodiesV G,
                                                           const float4* __restrict__ wa, const float4* __restrict__ wb,
                                                           float* acc_jn, float2* acc_jt, int iters, float tol,
                                                           uint32_t* stats, const uint32_t* __restrict__ row_islid,
                                                           uint32_t* isl_final) {
  if (blockIdx.x >= n_listed) return;
  const uint32_t g = glist[blockIdx.x];
  if (g_class[g] != want_class) return;
  extern __shared__ float4 big_raw[];
  BigStage<CH>* stg = reinterpret_cast<BigStage<CH>*>(big_raw);
  float4* lin = reinterpret_cast<float4*>(stg + 2);
  float4* ang = lin + BC;
  uint32_t* lvl = reinterpret_cast<uint32_t*>(ang + BC);
  __shared__ uint32_t res_bits;
  const uint32_t tid = threadIdx.x;
  const uint32_t nbg = gb_cnt[g], b0 = gb_start[g];
  const uint32_t off = S.lvl_off[g], nl = S.nlev[g];
  if (nbg > BC || nl > LC) {  // not reached: the class was chosen by these sizes
    if (tid == 0) atomicOr(&stats[STAT_ERR], 2u);
    return;
  }
  for (uint32_t i = tid; i < nbg; i += CH) {
    uint32_t b = gb_list[b0 + i];
    lin[i] = G.lin[b];
    ang[i] = G.ang[b];
  }
  for (uint32_t L = tid; L <= nl; L += CH) lvl[L] = S.lvl_start[off + L];
  if (tid == 0) res_bits = 0u;
  __syncthreads();
  // warm start application, level by level, rows read directly (one pass)
  for (uint32_t L = 0; L < nl; ++L) {
    for (uint32_t s = lvl[L] + tid; s < lvl[L + 1]; s += CH) {
      int e = R.wm[s];
      float4 pr = R.pred[s];
      if (e < 0 && pr.w == 0.0f && !(R.flags[s] & RF_JWARM)) continue;
      SRow r = ld_srow(R, s);
      const float4* x = X + 7 * (size_t)s;
      float q[24];
      for (int k = 0; k < 6; ++k) { float4 v = x[k]; q[4 * k] = v.x; q[4 * k + 1] = v.y; q[4 * k + 2] = v.z; q[4 * k + 3] = v.w; }
      m3 qa = mcols(mk3(q[0], q[1], q[2]), mk3(q[3], q[4], q[5]), mk3(q[6], q[7], q[8]));
      m3 qb = mcols(mk3(q[12], q[13], q[14]), mk3(q[15], q[16], q[17]), mk3(q[18], q[19], q[20]));
      float jn = 0.0f; float2 jt = make_float2(0.0f, 0.0f);
      if (warm_select(lin, ang, r, qa, qb, q[9], q[21], e >= 0, e >= 0 ? wa[e] : make_float4(0, 0, 0, 0),
                      e >= 0 ? wb[e] : make_float4(0, 0, 0, 0), pr, jn, jt))
        atomicAdd(&stats[STAT_PRED_USED], 1u);
      J[s] = make_float4(jn, jt.x, jt.y, 0.0f);
    }
    __threadfence_block();
    __syncthreads();
  }
  // sweeps: chunk (L, c0, c1) -> the next chunk of this sweep, or the first one of the next
  uint32_t cL = 0, c0 = lvl[0], c1 = min(lvl[0] + (uint32_t)CH, lvl[1]);
  int it = 0, buf = 0;
  big_stage_issue(stg[0], c0, c1 - c0, R, X, J);
  cp_async_commit();
  bool done = nl == 0;
  while (!done) {
    uint32_t nL = cL, n0, n1;
    bool last_of_sweep = false;
    if (c1 < lvl[cL + 1]) { n0 = c1; n1 = min(c1 + (uint32_t)CH, lvl[cL + 1]); }
    else if (cL + 1 < nl) { nL = cL + 1; n0 = lvl[nL]; n1 = min(n0 + (uint32_t)CH, lvl[nL + 1]); }
    else { last_of_sweep = true; nL = 0; n0 = lvl[0]; n1 = min(n0 + (uint32_t)CH, lvl[1]); }
    // a sweep of one chunk would prefetch the rows it is about to write: stage those after it
    const bool self_next = n0 == c0;
    if (!self_next) big_stage_issue(stg[buf ^ 1], n0, n1 - n0, R, X, J);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    if (tid < c1 - c0) {
      BigStage<CH>& st = stg[buf];
      m3 qa, qb; float ima, imb;
      SRow r = big_row(st, tid, &qa, &qb, &ima, &imb);
      // a joint is one unit: its first row runs all its rows in order (the later ones from global)
      const bool skip = (r.flags & RF_JOINT) && !(r.flags & RF_JFIRST);
      const uint32_t cnt = (r.flags & RF_JOINT) ? (uint32_t)r.t1.x : 1u;
      float rr = 0.0f;
      for (uint32_t q = 0; q < cnt && !skip; ++q) {
        const uint32_t sq = c0 + tid + q;
        if (q) r = big_row_global(R, X, sq, &qa, &qb, &ima, &imb);
        float4 jj = q ? J[sq] : st.j[tid];
        float jn = jj.x; float2 jt = make_float2(jj.y, jj.z);
        float d3[3];
        pgs_row_core(lin, ang, r, qa, qb, ima, imb, jn, jt, d3);
        J[sq] = make_float4(jn, jt.x, jt.y, 0.0f);
        if (r.m_n > 0.0f) rr = rmax(rr, fabsf(d3[0]) / r.m_n);
        if (r.m_t1 > 0.0f) rr = rmax(rr, fabsf(d3[1]) / r.m_t1);
        if (r.m_t2 > 0.0f) rr = rmax(rr, fabsf(d3[2]) / r.m_t2);
      }
      atomicMax(&res_bits, fbits(rr));  // non-negative floats: integer max, order-free
    }
    __threadfence_block();
    __syncthreads();
    if (self_next) {
      big_stage_issue(stg[buf ^ 1], n0, n1 - n0, R, X, J);
      cp_async_commit();
    }
    if (last_of_sweep) {
      it++;
      uint32_t rb = res_bits;
      __syncthreads();
      if (tid == 0) res_bits = 0u;
      if ((tol > 0.0f && __uint_as_float(rb) <= tol) || it >= iters) {
        done = true;
        if (tid == 0) {
          atomicMax(&stats[STAT_SWEEPS], (uint32_t)it);
          atomicMax(&stats[STAT_RESID], rb);
          atomicAdd(&stats[STAT_ROWSWEEPS], (lvl[nl] - lvl[0]) * (uint32_t)it);
          isl_final[row_islid[S.ord[lvl[0]]]] = rb;  // the group is one island
          if (tol > 0.0f && !(__uint_as_float(rb) <= tol)) {
            atomicAdd(&stats[STAT_ISLANDS_CAPPED], 1u);
            atomicAdd(&stats[STAT_ROWS_CAPPED], lvl[nl] - lvl[0]);
          }
        }
      }
      __syncthreads();
    }
    cL = nL; c0 = n0; c1 = n1; buf ^= 1;
  }
  cp_async_wait0();
  __syncthreads();
  for (uint32_t i = tid; i < nbg; i += CH) {
    uint32_t b = gb_list[b0 + i];
    G.lin[b] = lin[i];
    G.ang[b] = ang[i];
  }
  for (uint32_t s = lvl[0] + tid; s < lvl[nl]; s += CH) {
    uint32_t r = S.ord[s];
    float4 jj = J[s];
    acc_jn[r] = jj.x;
    acc_jt[r] = make_float2(jj.y, jj.z);
  }
}

// ------------------------------------------------------------------ learned warm start: features
// 24 features per scheduled contact row (rows with no movable body stay invalid), in the
// impulse unit u = m_n * kImpulseUnit where impulses appear:
//   0-2 normal; 3-5 relative linear velocity (B - A); 6-8 relative angular velocity (B - A);
//   9 depth x 10; 10-11 inverse masses x m_n; 12-14 A's angular response along n, t1, t2
//   ((r x d) . Iw (r x d)) x m_n; 15-17 the same for B; 18 static friction; 19-21 the previous
//   tick's impulse (normal, t1, t2) / u, 0 when cold; 22 1 when a previous impulse matched;
//   23 depth bias x 0.1.
__device__ __forceinline__ float ang_resp(const float* Iw, f3 r, f3 d) {
  m3 M = mcols(mk3(Iw[0], Iw[1], Iw[2]), mk3(Iw[3], Iw[4], Iw[5]), mk3(Iw[6], Iw[7], Iw[8]));
  f3 c = cross(r, d);
  return dot(c, mvec(M, c));
}
__global__ void k_row_features(uint32_t nc, RowsV R, BodiesV B, const float4* __restrict__ c_pt,
                               const int* __restrict__ wm_idx, const float4* __restrict__ wa, const float4* __restrict__ wb,
                               float* feat, uint8_t* valid) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  float* f = feat + 24 * (size_t)k;
  uint32_t fl = R.flags[k];
  if (!(fl & (RF_WA | RF_WB))) { valid[k] = 0; for (int q = 0; q < 24; ++q) f[q] = 0.0f; return; }
  valid[k] = 1;
  uint2 ab = R.ab[k];
  const bool terr = fl & RF_TERRAIN;
  float4 ra = R.ra[k], rb = R.rb[k], n4 = R.n[k], t14 = R.t1[k], t24 = R.t2[k];
  f3 n = xyz(n4), t1 = xyz(t14), t2 = xyz(t24);
  float mn = ra.w, u = mn > 0.0f ? mn * kImpulseUnit : 1.0f;
  float2 iv = R.inv[k];
  f3 la = xyz(B.lin[ab.x]), aa = xyz(B.ang[ab.x]);
  f3 lb = terr ? mk3(0, 0, 0) : xyz(B.lin[ab.y]), abv = terr ? mk3(0, 0, 0) : xyz(B.ang[ab.y]);
  f3 dl = lb - la, da = abv - aa;
  f[0] = n.x; f[1] = n.y; f[2] = n.z;
  f[3] = dl.x; f[4] = dl.y; f[5] = dl.z;
  f[6] = da.x; f[7] = da.y; f[8] = da.z;
  f[9] = c_pt[k].w * 10.0f;
  f[10] = iv.x * mn; f[11] = iv.y * mn;
  for (int q = 12; q < 18; ++q) f[q] = 0.0f;
  if (iv.x > 0.0f) {
    const float* I = B.Iw + 9 * (size_t)ab.x;
    f[12] = ang_resp(I, xyz(ra), n) * mn; f[13] = ang_resp(I, xyz(ra), t1) * mn; f[14] = ang_resp(I, xyz(ra), t2) * mn;
  }
  if (iv.y > 0.0f) {
    const float* I = B.Iw + 9 * (size_t)ab.y;
    f[15] = ang_resp(I, xyz(rb), n) * mn; f[16] = ang_resp(I, xyz(rb), t1) * mn; f[17] = ang_resp(I, xyz(rb), t2) * mn;
  }
  f[18] = R.mu[k].x;
  int e = wm_idx[k];
  if (e >= 0) {
    f3 jt = xyz(wb[e]);
    f[19] = wa[e].w / u; f[20] = dot(jt, t1) / u; f[21] = dot(jt, t2) / u; f[22] = 1.0f;
  } else {
    f[19] = f[20] = f[21] = 0.0f; f[22] = 0.0f;
  }
  f[23] = t14.w * 0.1f;
}
// The rows' converged impulses after the velocity sweeps, in the same unit (training targets).
__global__ void k_row_targets(uint32_t nc, RowsV R, const float* __restrict__ acc_jn, const float2* __restrict__ acc_jt,
                              float* t) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nc) return;
  float mn = R.ra[k].w, u = mn > 0.0f ? mn * kImpulseUnit : 1.0f;
  float2 jt = acc_jt[k];
  t[3 * k] = acc_jn[k] / u; t[3 * k + 1] = jt.x / u; t[3 * k + 2] = jt.y / u;
}

// ------------------------------------------------------------------ small helpers
__global__ void k_scatter_u32(uint32_t n, const uint32_t* __restrict__ idx, const uint32_t* __restrict__ src, uint32_t* dst) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[idx[i]] = src[i];
}
__global__ void k_flag_sched(uint32_t n, const uint32_t* __restrict__ root, uint8_t* fl) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) fl[k] = root[k] != 0xFFFFFFFFu;
}
__global__ void k_run_starts(uint32_t n, const uint32_t* __restrict__ roots, uint32_t* start_flag) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n) start_flag[s] = (s == 0 || roots[s] != roots[s - 1]) ? 1u : 0u;
}
__global__ void k_island_starts(uint32_t n, const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                                uint32_t* isl_start) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n && flag[s]) isl_start[pos[s]] = s;
}
__global__ void k_island_counts(uint32_t nisl, uint32_t n, const uint32_t* __restrict__ isl_start, uint32_t* isl_cnt) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nisl) isl_cnt[i] = (i + 1 < nisl ? isl_start[i + 1] : n) - isl_start[i];
}
__global__ void k_warm_merge_kept(uint32_t n, const uint4* __restrict__ kk, const float4* __restrict__ ka,
                                  const float4* __restrict__ kb, const uint4* __restrict__ newk, uint32_t n_new, uint4* ok,
                                  float4* oa, float4* ob) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  uint32_t p = j + key_lower_bound(newk, n_new, kk[j]);
  ok[p] = kk[j]; oa[p] = ka[j]; ob[p] = kb[j];
}

// Rows of the position-pass schedule: contacts, and each joint's first row.
__global__ void k_pos_keep(uint32_t n, uint32_t nc, const uint32_t* __restrict__ rows, const uint32_t* __restrict__ flags,
                           uint8_t* keep) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t r = rows[i];
  keep[i] = (r < nc || (flags[r] & RF_JFIRST)) ? 1 : 0;
}
// Position i of the scheduled-row scan: joint rows (index nc .. nc + njr) first, then the contacts;
// the row there and whether it is scheduled (a root was found for it).
__global__ void k_joint_first_order(uint32_t n, uint32_t nc, uint32_t njr, const uint32_t* __restrict__ root,
                                    uint32_t* idx, uint8_t* fl) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t r = i < njr ? nc + i : i - njr;
  idx[i] = r;
  fl[i] = root[r] != 0xFFFFFFFFu ? 1 : 0;
}
// ------------------------------------------------------------------ host driver
// Replaces a built level schedule (ord sorted by (group, level), level starts, level counts, the
// level histogram and each row's level) by the coloured one (k_colour_levels): rows sorted by
// (group, colour), stable, so a colour's rows keep their (level, serial) order.
static void colour_schedule(WorldGpu::Scratch& S, uint32_t nsched, uint32_t ng, uint32_t g_small, uint32_t nb, const uint32_t* g_start,
                            const uint32_t* g_cnt, DBuf<uint32_t>& ord, DBuf<uint32_t>& lvl_off, DBuf<uint32_t>& lvl_start,
                            DBuf<uint32_t>& nlev, uint32_t* hist, uint32_t* row_level, cudaStream_t st) {
  if (!nsched || !ng) return;
  S.col_mask.ensure(nb + 1);
  S.col_nlev.ensure(ng + 1);
  S.col_ord.ensure(nsched + 1);
  S.key64.ensure(nsched + 1); S.key64b.ensure(nsched + 1);
  RP_CUDA(cudaMemsetAsync(S.col_mask.p, 0, sizeof(uint4) * (size_t)(nb + 1), st));
  k_colour_levels<<<nblk(ng * 32, 128), 128, 0, st>>>(ng, g_small, ord.p, lvl_off.p, lvl_start.p, nlev.p, S.r_ab.p, S.r_flags.p,
                                                      S.col_mask.p, S.key64.p, S.col_nlev.p); RP_COUNT_LAUNCH(1);
  sort_pairs_u64(S, S.key64.p, S.key64b.p, ord.p, S.col_ord.p, nsched, 0, 64, st);
  RP_CUDA(cudaMemcpyAsync(ord.p, S.col_ord.p, sizeof(uint32_t) * (size_t)nsched, cudaMemcpyDeviceToDevice, st));
  RP_CUDA(cudaMemcpyAsync(nlev.p, S.col_nlev.p, sizeof(uint32_t) * (size_t)ng, cudaMemcpyDeviceToDevice, st));
  S.lv_np1.ensure(ng + 1);
  k_plus1<<<nblk(ng), T, 0, st>>>(ng, nlev.p, S.lv_np1.p); RP_COUNT_LAUNCH(1);
  uint32_t total = exclusive_scan_total(S, S.lv_np1.p, lvl_off.p, ng, st);
  lvl_start.ensure(total + 1);
  if (hist) RP_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * (size_t)(nsched + 1), st));
  k_level_starts<<<nblk(nsched), T, 0, st>>>(nsched, S.key64b.p, lvl_off.p, nlev.p, g_start, g_cnt, lvl_start.p, hist);
  RP_COUNT_LAUNCH(1);
  if (row_level) { k_row_key_level<<<nblk(nsched), T, 0, st>>>(nsched, ord.p, S.key64b.p, row_level); RP_COUNT_LAUNCH(1); }
}
// units: R.t1 of the rows when a joint's rows form one schedule unit (the velocity schedule), else null.
static void build_schedule(WorldGpu::Scratch& S, uint32_t* W_err, uint32_t nsched, uint32_t nisl, const uint32_t* ord_in,
                           const uint32_t* isl_start, const uint32_t* isl_cnt, uint32_t* ord_out, DBuf<uint32_t>& lvl_off,
                           DBuf<uint32_t>& lvl_start, DBuf<uint32_t>& nlev, uint32_t* hist, uint32_t* row_level,
                           cudaStream_t st, const float4* units = nullptr) {
  nlev.ensure(nisl + 1);
  lvl_off.ensure(nisl + 1);
  S.key64.ensure(nsched + 1); S.key64b.ensure(nsched + 1);
  // predecessors, then levels (see k_level_entries)
  S.lv_key.ensure(2 * (size_t)nsched + 2); S.lv_key2.ensure(2 * (size_t)nsched + 2);
  S.lv_val.ensure(2 * (size_t)nsched + 2); S.lv_val2.ensure(2 * (size_t)nsched + 2);
  S.lv_pred.ensure(2 * (size_t)nsched + 2); S.lv_level.ensure(nsched + 1);
  if (units) S.lv_lead.ensure(nsched + 1);
  uint32_t* lead = units ? S.lv_lead.p : nullptr;
  k_level_entries<<<nblk(nsched), T, 0, st>>>(nsched, ord_in, S.r_ab.p, S.r_flags.p, units, S.lv_key.p, S.lv_val.p, lead); RP_COUNT_LAUNCH(1);
  sort_pairs_u32(S, S.lv_key.p, S.lv_key2.p, S.lv_val.p, S.lv_val2.p, 2 * nsched, 0, 32, st);
  RP_CUDA(cudaMemsetAsync(S.lv_pred.p, 0xFF, sizeof(uint32_t) * 2 * (size_t)nsched, st));
  k_level_preds<<<nblk(2 * nsched), T, 0, st>>>(2 * nsched, S.lv_key2.p, S.lv_val2.p, S.lv_pred.p); RP_COUNT_LAUNCH(1);
  k_level_relax<<<nblk(nisl * 32, 128), 128, 0, st>>>(nisl, isl_start, isl_cnt, ord_in, S.lv_pred.p, lead, S.lv_level.p,
                                                      S.key64.p, nlev.p, row_level, W_err); RP_COUNT_LAUNCH(1);
  sort_pairs_u64(S, S.key64.p, S.key64b.p, ord_in, ord_out, nsched, 0, 64, st);
  S.lv_np1.ensure(nisl + 1);
  k_plus1<<<nblk(nisl), T, 0, st>>>(nisl, nlev.p, S.lv_np1.p); RP_COUNT_LAUNCH(1);
  uint32_t total = exclusive_scan_total(S, S.lv_np1.p, lvl_off.p, nisl, st);
  lvl_start.ensure(total + 1);
  k_level_starts<<<nblk(nsched), T, 0, st>>>(nsched, S.key64b.p, lvl_off.p, nlev.p, isl_start, isl_cnt, lvl_start.p,
                                             hist); RP_COUNT_LAUNCH(1);
}

// The W6 passes' scratch: per body, per contact, and a fixed pool for the direct solves.
static w6::W6V w6_view(WorldGpu::Scratch& S) {
  w6::W6V V;
  V.rest_cnt = S.w6_rest_cnt.p; V.rest_min = S.w6_rest_min.p; V.rest_max = S.w6_rest_max.p;
  V.parent = S.w6_parent.p; V.slot = S.w6_slot.p;
  V.involved = S.w6_involved.p; V.direct = S.w6_direct.p; V.in_set = S.w6_in_set.p; V.has_pseudo = S.w6_has_pseudo.p;
  V.acc = S.w6_acc.p; V.pl = S.w6_pl.p; V.pa = S.w6_pa.p;
  V.rows = S.w6_rows.p; V.target = S.w6_target.p; V.sup_acc = S.w6_sup_acc.p; V.pseudo_u = S.w6_pseudo_u.p;
  V.comp_rows = S.w6_comp_rows.p; V.comp_start = S.w6_comp_start.p; V.row_comp = S.w6_row_comp.p; V.cur = S.w6_cur.p;
  V.ctr = S.w6_ctr.p;
  V.pool = S.w6_pool.p;
  V.pool_bytes = S.w6_pool.cap;
  V.toi_a = S.toi_a.p; V.toi_b = S.toi_b.p;
  return V;
}
static constexpr size_t kW6Pool = 48ull << 20;  // direct-solve scratch: about eleven 250-row components at once

void run_solve(WorldGpu& W, StepCtx& ctx) {
  auto& S = *W.s_;
  cudaStream_t st = W.stream();
  const uint32_t nb = W.num_bodies(), nc = ctx.nc;
  uint32_t* stats = W.d_stats.p;
  W.pred_valid_ = false;
  // joints: their rows follow the contact rows in the row arrays (index nc + r)
  const uint32_t nj = W.num_joints();
  const uint8_t* jointed = nj ? W.jointed_d.p : nullptr;
  uint32_t njr = 0, npp = 0;  // joint rows; rows of the position-pass schedule (0: the main one)
  uint32_t cls_n[32] = {};    // solve groups per class (class 3: g_small, not listed)
  S.constrained.ensure(nb + 1); S.loaded.ensure(nb + 1); S.ballistic.ensure(nb + 1); S.touching.ensure(nb + 1);
  S.uf.ensure(nb + 1); S.uf2.ensure(nb + 1); S.body_level.ensure(nb + 1); S.root_mark.ensure(nb + 1);
  S.Iw.ensure(9 * (size_t)nb + 9);
  S.orig_pos.ensure(nb + 1); S.orig_rot.ensure(nb + 1); S.pred_pos.ensure(nb + 1); S.pred_rot.ensure(nb + 1);
  S.split_l.ensure(nb + 1); S.split_a.ensure(nb + 1);
  S.toi_a.ensure(nc + 1); S.toi_b.ensure(nc + 1);
  S.w6_rest_cnt.ensure(nb + 1); S.w6_rest_min.ensure(nb + 1); S.w6_rest_max.ensure(nb + 1); S.w6_parent.ensure(nb + 1);
  S.w6_slot.ensure(nb + 1); S.w6_involved.ensure(nb + 1); S.w6_direct.ensure(nb + 1); S.w6_acc.ensure(6 * (size_t)nb + 6);
  S.w6_pl.ensure(nb + 1); S.w6_pa.ensure(nb + 1);
  S.w6_rows.ensure(nc + 1); S.w6_target.ensure(nc + 1); S.w6_sup_acc.ensure(nc + 1); S.w6_pseudo_u.ensure(nc + 1);
  S.w6_in_set.ensure(nc + 1); S.w6_has_pseudo.ensure(nc + 1); S.w6_comp_rows.ensure(nc + 1);
  S.w6_comp_start.ensure(nc + 2); S.w6_row_comp.ensure(nc + 1); S.w6_cur.ensure(nc + 1);
  S.w6_ctr.ensure(w6::C_N); S.w6_pool.ensure(kW6Pool);
  RP_CUDA(cudaMemsetAsync(S.w6_ctr.p, 0, sizeof(uint32_t) * w6::C_N, st));  // no bounce until the count says so
  RP_CUDA(cudaMemsetAsync(S.loaded.p, 0, nb + 1, st));
  RP_CUDA(cudaMemsetAsync(S.constrained.p, 0, nb + 1, st));
  RP_CUDA(cudaMemsetAsync(S.touching.p, 0, nb + 1, st));
  RP_CUDA(cudaMemsetAsync(S.split_l.p, 0, sizeof(float4) * (nb + 1), st));
  RP_CUDA(cudaMemsetAsync(S.split_a.p, 0, sizeof(float4) * (nb + 1), st));
  BodiesV B{W.pos.p, W.rot.p, W.lin.p, W.ang.p, W.inv_mass.p, S.Iw.p, W.inv_I.p, W.awake.p, W.dyn.p};
  RowsV R{S.r_ab.p, S.r_flags.p, S.r_inv.p, S.r_ra.p, S.r_rb.p, S.r_n.p, S.r_t1.p, S.r_t2.p, S.r_mu.p, S.r_la.p};
  ctx.nisl = 0;
  auto& P = S.prof;
  P.begin(PH_ISLANDS, st);
  // ---- the reference's islands: their count, and whether the solve runs (step.rs:146-150)
  uint32_t nref = 0;
  if ((nc > 0 || nj > 0) && nb > 0) {
    k_iota<<<nblk(nb), T, 0, st>>>(nb, S.uf2.p); RP_COUNT_LAUNCH(1);
    RP_CUDA(cudaMemsetAsync(S.root_mark.p, 0, sizeof(uint32_t) * nb, st));
    joints_ref_islands(W, S.uf2.p, nullptr, true, st);
    if (nc) {
      k_union_contacts<<<nblk(nc), T, 0, st>>>(nc, 0, S.c_a.p, S.c_b.p, W.col_body.p, W.inv_mass.p, W.awake.p, nullptr,
                                               S.uf2.p); RP_COUNT_LAUNCH(1);
      k_ref_island_marks<<<nblk(nc), T, 0, st>>>(nc, S.c_a.p, S.c_b.p, W.col_body.p, W.inv_mass.p, S.uf2.p, S.root_mark.p); RP_COUNT_LAUNCH(1);
    }
    joints_ref_islands(W, S.uf2.p, S.root_mark.p, false, st);
    S.tmp32.ensure(nb + 1);
    nref = exclusive_scan_total(S, S.root_mark.p, S.tmp32.p, nb, st);
  }
  ctx.nref_isl = nref;
  W.st_.islands = nref;
  S.row_level.ensure(nc + 1);
  RP_CUDA(cudaMemsetAsync(S.row_level.p, 0xFF, sizeof(uint32_t) * (nc + 1), st));
  W.levels_valid_ = true;
  P.end(PH_ISLANDS, st);
  if (nref > 0) {
    // ---- rows
    P.begin(PH_ROWS, st);
    k_world_inertia<<<nblk(nb), T, 0, st>>>(nb, W.rot.p, W.inv_mass.p, W.inv_I.p, S.Iw.p); RP_COUNT_LAUNCH(1);
    njr = joints_count_rows(W, ctx.dt, B, st);
    const uint32_t nall = nc + njr;
    if (njr) {  // the level of every scheduled row is written, joint rows included
      S.row_level.ensure(nall + 1);
      RP_CUDA(cudaMemsetAsync(S.row_level.p, 0xFF, sizeof(uint32_t) * (nall + 1), st));
    }
    S.r_ab.ensure(nall + 1); S.r_flags.ensure(nall + 1); S.r_inv.ensure(nall + 1); S.r_ra.ensure(nall + 1);
    S.r_rb.ensure(nall + 1); S.r_n.ensure(nall + 1); S.r_t1.ensure(nall + 1); S.r_t2.ensure(nall + 1);
    S.r_mu.ensure(nall + 1); S.r_la.ensure(nall + 1); S.acc_jn.ensure(nall + 1); S.acc_jt.ensure(nall + 1);
    S.wm_idx.ensure(nc + 1); S.row_isl.ensure(nall + 1); S.row_isl2.ensure(nall + 1);
    R = RowsV{S.r_ab.p, S.r_flags.p, S.r_inv.p, S.r_ra.p, S.r_rb.p, S.r_n.p, S.r_t1.p, S.r_t2.p, S.r_mu.p, S.r_la.p};
    // solve islands: joint rows, then contacts (a sleeping jointed side counts), then every row's root
    k_iota<<<nblk(nb), T, 0, st>>>(nb, S.uf.p); RP_COUNT_LAUNCH(1);
    joints_build_rows(W, ctx.dt, B, R, nc, S.acc_jn.p, S.acc_jt.p, S.uf.p, st);
    if (nc) {
      k_union_contacts<<<nblk(nc), T, 0, st>>>(nc, 1, S.c_a.p, S.c_b.p, W.col_body.p, W.inv_mass.p, W.awake.p, jointed,
                                               S.uf.p); RP_COUNT_LAUNCH(1);
      k_build_rows<<<nblk(nc), T, 0, st>>>(nc, ctx.dt, S.c_a.p, S.c_b.p, S.c_pt.p, S.c_n.p, W.col_body.p, W.col_mat.p,
                                           ctx.hf_mat, W.pair_table.p, B, S.pre_lin.p, S.pre_ang.p, R, S.acc_jn.p,
                                           S.acc_jt.p, S.uf.p, S.row_isl.p, jointed, W.last_lin.p, S.toi_a.p,
                                           S.toi_b.p); RP_COUNT_LAUNCH(1);
    }
    joints_row_roots(W, R, nc, njr, S.uf.p, S.row_isl.p, st);
    P.end(PH_ROWS, st);
    P.begin(PH_SCHED, st);
    // ---- solve islands: roots of scheduled rows -> dense island ids, rows grouped by island
    S.flag8.ensure(nall + 1); S.rows_sched.ensure(nall + 1); S.rows_sched2.ensure(nall + 1);
    S.tmp32.ensure(nall + 1); S.tmp32b.ensure(nall + 1);
    uint32_t nsched = 0;
    // scheduled rows in the order joint rows, then contacts: the stable sort by island below keeps
    // every island's joint rows ahead of its contacts
    k_joint_first_order<<<nblk(nall), T, 0, st>>>(nall, nc, njr, S.row_isl.p, S.tmp32b.p, S.flag8.p); RP_COUNT_LAUNCH(1);
    {
      size_t bytes = 0;
      S.counts.ensure(4);
      RP_CUDA(cub::DeviceSelect::Flagged(nullptr, bytes, S.tmp32b.p, S.flag8.p, S.rows_sched.p, S.counts.p + 3, nall, st));
      S.cub_tmp.ensure(bytes + 16);
      RP_CUDA(cub::DeviceSelect::Flagged(S.cub_tmp.p, bytes, S.tmp32b.p, S.flag8.p, S.rows_sched.p, S.counts.p + 3, nall, st));
      RP_COUNT_LAUNCH(2);
      RP_CUDA(cudaMemcpyAsync(&nsched, S.counts.p + 3, 4, cudaMemcpyDeviceToHost, st));
      RP_CUDA(cudaStreamSynchronize(st));
    }
    ctx.nsched = nsched;
    uint32_t nisl = 0, ng = 0, g_small = 0;
    S.isl_start.ensure(nsched + 1); S.isl_cnt.ensure(nsched + 1);
    S.ord_main.ensure(nsched + 1); S.ord_vs.ensure(nsched + 1); S.ord_ps.ensure(nsched + 1);
    if (nsched > 0) {
      // island root per scheduled row; sorting (root, row) makes each island's rows contiguous, in order
      k_gather_u32<<<nblk(nsched), T, 0, st>>>(nsched, S.rows_sched.p, S.row_isl.p, S.tmp32.p); RP_COUNT_LAUNCH(1);
      sort_pairs_u32(S, S.tmp32.p, S.tmp32b.p, S.rows_sched.p, S.rows_sched2.p, nsched, 0, 32, st);
      S.woff.ensure(nsched + 1); S.wpos.ensure(nsched + 1);
      k_run_starts<<<nblk(nsched), T, 0, st>>>(nsched, S.tmp32b.p, S.woff.p); RP_COUNT_LAUNCH(1);
      nisl = exclusive_scan_total(S, S.woff.p, S.wpos.p, nsched, st);
      k_island_starts<<<nblk(nsched), T, 0, st>>>(nsched, S.woff.p, S.wpos.p, S.isl_start.p); RP_COUNT_LAUNCH(1);
      k_island_counts<<<nblk(nisl), T, 0, st>>>(nisl, nsched, S.isl_start.p, S.isl_cnt.p); RP_COUNT_LAUNCH(1);
      // ---- solve groups: small islands packed by the prefix sum of their rows, big ones alone
      S.g_small_rows.ensure(nisl + 1); S.g_small_pre.ensure(nisl + 1); S.g_big.ensure(nisl + 1);
      S.g_big_pre.ensure(nisl + 1); S.g_of_isl.ensure(nisl + 1);
      const uint32_t group_rows = W.tuning_.group_rows;
      k_group_flags<<<nblk(nisl), T, 0, st>>>(nisl, group_rows, S.isl_cnt.p, S.g_small_rows.p, S.g_big.p); RP_COUNT_LAUNCH(1);
      // small islands are packed in order of their row count (island order among equal counts), so
      // a group holds islands of about one size: a small island is mostly a chain of rows on one
      // body, so its levels are about its rows, and a group's levels are its deepest island's
      S.g_iota.ensure(nisl + 1); S.g_perm.ensure(nisl + 1); S.g_sz_sorted.ensure(nisl + 1); S.g_pre_sorted.ensure(nisl + 1);
      k_iota<<<nblk(nisl), T, 0, st>>>(nisl, S.g_iota.p); RP_COUNT_LAUNCH(1);
      int sbits = 1;
      while ((1u << sbits) <= group_rows) sbits++;
      sort_pairs_u32(S, S.g_small_rows.p, S.g_sz_sorted.p, S.g_iota.p, S.g_perm.p, nisl, 0, sbits, st);
      uint32_t small_total = exclusive_scan_total(S, S.g_sz_sorted.p, S.g_pre_sorted.p, nisl, st);
      k_scatter_u32<<<nblk(nisl), T, 0, st>>>(nisl, S.g_perm.p, S.g_pre_sorted.p, S.g_small_pre.p); RP_COUNT_LAUNCH(1);
      uint32_t nbig = exclusive_scan_total(S, S.g_big.p, S.g_big_pre.p, nisl, st);
      g_small = small_total ? (small_total - 1) / group_rows + 1 : 0;
      ng = g_small + nbig;
      k_group_of_isl<<<nblk(nisl), T, 0, st>>>(nisl, group_rows, S.isl_cnt.p, S.g_small_pre.p, S.g_big_pre.p, g_small,
                                                S.g_of_isl.p); RP_COUNT_LAUNCH(1);
      S.g_key.ensure(nsched + 1); S.g_key2.ensure(nsched + 1);
      k_group_keys<<<nblk(nsched), T, 0, st>>>(nsched, S.woff.p, S.wpos.p, S.g_of_isl.p, S.g_key.p); RP_COUNT_LAUNCH(1);
      int gbits = 1;
      while ((1u << gbits) < ng + 1 && gbits < 32) gbits++;
      sort_pairs_u32(S, S.g_key.p, S.g_key2.p, S.rows_sched2.p, S.tmp32.p, nsched, 0, gbits, st);  // rows by group, stable
      S.g_start.ensure(ng + 1); S.g_cnt.ensure(ng + 1); S.g_class.ensure(ng + 1);
      RP_CUDA(cudaMemsetAsync(S.g_start.p, 0, sizeof(uint32_t) * (ng + 1), st));
      RP_CUDA(cudaMemsetAsync(S.g_cnt.p, 0, sizeof(uint32_t) * (ng + 1), st));
      k_group_ranges<<<nblk(nsched), T, 0, st>>>(nsched, S.g_key2.p, S.g_start.p, S.g_cnt.p); RP_COUNT_LAUNCH(1);
      S.row_isl2.ensure(nall + 1);
      k_scatter_u32<<<nblk(nsched), T, 0, st>>>(nsched, S.tmp32.p, S.g_key2.p, S.row_isl2.p); RP_COUNT_LAUNCH(1);  // group of each row
      // each row's island inside its group (the per-island residual stop)
      S.row_islid.ensure(nall + 1); S.row_lisl.ensure(nall + 1); S.li_flag.ensure(nsched + 1); S.li_pre.ensure(nsched + 1);
      S.g_nisl.ensure(ng + 1);
      k_row_island<<<nblk(nsched), T, 0, st>>>(nsched, S.rows_sched2.p, S.woff.p, S.wpos.p, S.row_islid.p); RP_COUNT_LAUNCH(1);
      k_local_isl_flags<<<nblk(nsched), T, 0, st>>>(nsched, S.tmp32.p, S.g_key2.p, S.row_islid.p, S.li_flag.p); RP_COUNT_LAUNCH(1);
      exclusive_scan(S, S.li_flag.p, S.li_pre.p, nsched, st);
      k_local_isl<<<nblk(nsched), T, 0, st>>>(nsched, S.tmp32.p, S.g_key2.p, S.g_start.p, S.g_cnt.p, S.li_flag.p, S.li_pre.p,
                                              S.row_lisl.p, S.g_nisl.p); RP_COUNT_LAUNCH(1);
      ctx.nisl = ng;
      ctx.g_small = g_small;
      // ---- main schedule (row order within each group)
      S.lvl_hist.ensure(nsched + 1);
      RP_CUDA(cudaMemsetAsync(S.lvl_hist.p, 0, sizeof(uint32_t) * (nsched + 1), st));
      build_schedule(S, stats + STAT_ERR, nsched, ng, S.tmp32.p, S.g_start.p, S.g_cnt.p, S.ord_main.p, S.lvl_off, S.lvl_start,
                     S.nlev, S.lvl_hist.p, S.row_level.p, st, njr ? S.r_t1.p : nullptr);
      // coloured order (worlds without joints): every pass on the main schedule -- warm start,
      // sweeps, ballistic test, position projection -- then runs colour by colour
      if (W.coloured_ && njr == 0)
        colour_schedule(S, nsched, ng, g_small, nb, S.g_start.p, S.g_cnt.p, S.ord_main, S.lvl_off, S.lvl_start, S.nlev,
                        S.lvl_hist.p, S.row_level.p, st);
      // ---- the bodies each group moves, with their index inside the group
      S.body_grp.ensure(nb + 1); S.gb_tmp.ensure(nb + 1); S.gb_key.ensure(nb + 1); S.gb_key2.ensure(nb + 1);
      S.gb_list.ensure(nb + 1); S.gb_start.ensure(ng + 1); S.gb_cnt.ensure(ng + 1); S.body_local.ensure(nb + 1);
      RP_CUDA(cudaMemsetAsync(S.body_grp.p, 0xFF, sizeof(uint32_t) * (nb + 1), st));
      k_body_groups<<<nblk(nsched), T, 0, st>>>(nsched, S.tmp32.p, S.g_key2.p, S.r_ab.p, S.r_flags.p, S.body_grp.p); RP_COUNT_LAUNCH(1);
      // ---- the position pass's own schedule when there are joints: the contacts and one unit per
      // joint (its first row carries the joint's whole solve), in the same order -- without the
      // joints' other velocity rows, which would only add levels
      npp = 0;
      if (njr) {
        S.pp_rows.ensure(nsched + 1); S.pp_key.ensure(nsched + 1); S.pp_gs.ensure(ng + 1); S.pp_gc.ensure(ng + 1);
        S.ord_pp.ensure(nsched + 1);  // build_schedule's order output (it sizes the level arrays itself)
        S.flag8.ensure(nsched + 1);
        k_pos_keep<<<nblk(nsched), T, 0, st>>>(nsched, nc, S.tmp32.p, S.r_flags.p, S.flag8.p); RP_COUNT_LAUNCH(1);
        npp = select_flagged_u32(S, S.tmp32.p, S.flag8.p, S.pp_rows.p, nsched, st);
        select_flagged_u32(S, S.g_key2.p, S.flag8.p, S.pp_key.p, nsched, st);
        RP_CUDA(cudaMemsetAsync(S.pp_gs.p, 0, sizeof(uint32_t) * (ng + 1), st));
        RP_CUDA(cudaMemsetAsync(S.pp_gc.p, 0, sizeof(uint32_t) * (ng + 1), st));
        k_group_ranges<<<nblk(npp), T, 0, st>>>(npp, S.pp_key.p, S.pp_gs.p, S.pp_gc.p); RP_COUNT_LAUNCH(1);
        build_schedule(S, stats + STAT_ERR, npp, ng, S.pp_rows.p, S.pp_gs.p, S.pp_gc.p, S.ord_pp.p, S.lvl_off_pp,
                       S.lvl_start_pp, S.nlev_pp, nullptr, nullptr, st);
      }
      k_flag_grouped<<<nblk(nb), T, 0, st>>>(nb, S.body_grp.p, S.gb_key.p); RP_COUNT_LAUNCH(1);
      select_flagged_iota(S, nb, S.gb_key.p, S.gb_tmp.p, S.counts.p + 0, st);
      uint32_t ngb = 0;
      RP_CUDA(cudaMemcpyAsync(&ngb, S.counts.p + 0, 4, cudaMemcpyDeviceToHost, st));
      RP_CUDA(cudaStreamSynchronize(st));
      k_gather_u32<<<nblk(ngb), T, 0, st>>>(ngb, S.gb_tmp.p, S.body_grp.p, S.gb_key.p); RP_COUNT_LAUNCH(1);
      sort_pairs_u32(S, S.gb_key.p, S.gb_key2.p, S.gb_tmp.p, S.gb_list.p, ngb, 0, gbits, st);
      RP_CUDA(cudaMemsetAsync(S.gb_start.p, 0, sizeof(uint32_t) * (ng + 1), st));
      RP_CUDA(cudaMemsetAsync(S.gb_cnt.p, 0, sizeof(uint32_t) * (ng + 1), st));
      k_body_local<<<nblk(ngb), T, 0, st>>>(ngb, S.gb_key2.p, S.gb_list.p, S.gb_start.p, S.gb_cnt.p, S.body_local.p); RP_COUNT_LAUNCH(1);
      k_body_local2<<<nblk(ngb), T, 0, st>>>(ngb, S.gb_key2.p, S.gb_list.p, S.gb_start.p, S.body_local.p); RP_COUNT_LAUNCH(1);
      S.cls_cnt.ensure(32); S.cls_list.ensure(32 * (size_t)ng + 32);
      RP_CUDA(cudaMemsetAsync(S.cls_cnt.p, 0, 32 * 4, st));
      k_group_class<<<nblk(ng), T, 0, st>>>(ng, g_small, S.gb_cnt.p, S.g_cnt.p, S.nlev.p, S.g_class.p, S.cls_cnt.p,
                                            S.cls_list.p, stats); RP_COUNT_LAUNCH(1);
      RP_CUDA(cudaMemcpyAsync(cls_n, S.cls_cnt.p, 32 * 4, cudaMemcpyDeviceToHost, st));
      RP_CUDA(cudaStreamSynchronize(st));
      // levels / max batch (solver.rs:684-687)
      {
        size_t bytes = 0;
        RP_CUDA(cub::DeviceReduce::Max(nullptr, bytes, S.nlev.p, stats + STAT_LEVELS, ng, st));
        S.cub_tmp.ensure(bytes + 16);
        RP_CUDA(cub::DeviceReduce::Max(S.cub_tmp.p, bytes, S.nlev.p, stats + STAT_LEVELS, ng, st));
        RP_COUNT_LAUNCH(2);
        bytes = 0;
        RP_CUDA(cub::DeviceReduce::Max(nullptr, bytes, S.lvl_hist.p, stats + STAT_MAXBATCH, nsched, st));
        S.cub_tmp.ensure(bytes + 16);
        RP_CUDA(cub::DeviceReduce::Max(S.cub_tmp.p, bytes, S.lvl_hist.p, stats + STAT_MAXBATCH, nsched, st));
        RP_COUNT_LAUNCH(2);
      }
    }
    P.end(PH_SCHED, st);
    Sched SM{S.ord_main.p, S.lvl_off.p, S.lvl_start.p, S.nlev.p};
    P.begin(PH_WARM_MATCH, st);
    // ---- warm start matching (solver.rs:717-762)
    k_warm_match<<<nblk(nc), T, 0, st>>>(nc, S.r_ab.p, S.r_flags.p, S.r_la.p, W.warm_key.p, W.warm_a.p, W.n_warm,
                                         S.wm_idx.p, stats + STAT_WARM_MATCHED, stats + STAT_ERR); RP_COUNT_LAUNCH(1);
    if (njr && ng) { k_joint_warm<<<nblk(ng * 32, 128), 128, 0, st>>>(ng, nc, SM, R, B, S.acc_jn.p); RP_COUNT_LAUNCH(1); }
    k_warm_unscheduled<<<nblk(nc), T, 0, st>>>(nc, R, B, S.wm_idx.p, W.warm_a.p, W.warm_b.p, S.acc_jn.p, S.acc_jt.p); RP_COUNT_LAUNCH(1);
    // learned warm start: row features, and the model's prediction of every row's impulse
    const bool learned = W.model_ != nullptr;
    if (learned || W.feat_log_) {
      S.feat.ensure(24 * (size_t)nc + 24); S.feat_valid.ensure(nc + 1);
      k_row_features<<<nblk(nc), T, 0, st>>>(nc, R, B, S.c_pt.p, S.wm_idx.p, W.warm_a.p, W.warm_b.p, S.feat.p,
                                             S.feat_valid.p); RP_COUNT_LAUNCH(1);
    }
    if (learned) {
      S.pred3.ensure(3 * (size_t)nc + 3); S.pred_used.ensure(nc + 1);
      W.model_->predict_async(nc, S.feat.p, S.pred3.p, stats + STAT_ERR, st);  // no host wait mid-tick
    }
    W.pred_valid_ = learned;
    P.end(PH_WARM_MATCH, st);
    P.begin(PH_VEL_SOLVE, st);
    P.begin(PH_VEL_PREP, st);
    // ---- warm application + velocity sweeps
    const bool resid_mode = W.res_tol_ > 0.0f;
    int iters = (int)(resid_mode ? (W.res_max_ > 0 ? W.res_max_ : W.iters_v_) : W.iters_v_);
    if (ng > 0) {
      // rows in schedule order, then one CTA per group (bodies in shared memory); groups moving more
      // bodies than a CTA holds run on the warp kernel over global memory
      S.s_loc.ensure(nsched + 1); S.s_flags.ensure(nsched + 1); S.s_inv.ensure(nsched + 1); S.s_ra.ensure(nsched + 1);
      S.s_rb.ensure(nsched + 1); S.s_n.ensure(nsched + 1); S.s_t1.ensure(nsched + 1); S.s_t2.ensure(nsched + 1);
      S.s_mu.ensure(nsched + 1); S.s_va.ensure(nsched + 1); S.s_vb.ensure(nsched + 1); S.s_jn.ensure(nsched + 1);
      S.s_jt.ensure(nsched + 1); S.s_wm.ensure(nsched + 1); S.s_pred.ensure(nsched + 1);
      if (learned) RP_CUDA(cudaMemsetAsync(S.pred_used.p, 0, 16 * (size_t)nc, st));  // unscheduled rows: none
      SRowsV SR{S.s_loc.p, S.s_flags.p, S.s_inv.p, S.s_ra.p, S.s_rb.p, S.s_n.p, S.s_t1.p, S.s_t2.p, S.s_mu.p, S.s_va.p,
                S.s_vb.p, S.s_jn.p, S.s_jt.p, S.s_wm.p, S.s_pred.p};
      k_permute_rows<<<nblk(nsched), T, 0, st>>>(nsched, nc, S.ord_main.p, R, B, S.body_local.p, S.wm_idx.p, S.row_lisl.p,
                                                 learned ? S.pred3.p : nullptr, S.row_isl2.p, S.g_class.p,
                                                 learned ? S.pred_used.p : nullptr, W.pred_cold_only_ ? 1u : 0u, SR); RP_COUNT_LAUNCH(1);
      const float tol = resid_mode ? W.res_tol_ : 0.0f;
      S.isl_final.ensure(nisl + 1);
      // dynamic shared memory above the 48 KB default, opted into once per device
      const uint32_t gr = W.tuning_.group_rows;
      const OnchipLayout lay_packed = onchip_layout(WG_ROWS(gr), WG_BODIES(gr), WG_ROWS(gr));
      const OnchipLayout lay_packed_max = onchip_layout(WG_ROWS(GROUP_ROWS_MAX), WG_BODIES(GROUP_ROWS_MAX), WG_ROWS(GROUP_ROWS_MAX));
      const OnchipLayout lay_top = onchip_layout(kIslandRows[ISLAND_BUCKETS - 1], kIslandBodies[ISLAND_BUCKETS - 1], 1u);
      static std::atomic<unsigned long long> smem_attr{0};
      int dev = 0;
      RP_CUDA(cudaGetDevice(&dev));
      if (!((smem_attr.load() >> (dev & 63)) & 1ull)) {
        RP_CUDA(cudaFuncSetAttribute(k_vel_solve_big<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)big_smem<128>(kBigBodies[2], kBigLevels[2])));
        RP_CUDA(cudaFuncSetAttribute(k_vel_solve_big<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)big_smem<64>(kBigBodies[1], kBigLevels[1])));
        for (auto f : {k_vel_solve_onchip<false, 32>, k_vel_solve_onchip<false, 64>, k_vel_solve_onchip<false, 128>,
                       k_vel_solve_onchip<false, 256>})
          RP_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lay_top.bytes));
        for (auto f : {k_vel_solve_onchip<true, 32>, k_vel_solve_onchip<true, 64>, k_vel_solve_onchip<true, 128>})
          RP_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lay_packed_max.bytes));
        smem_attr.fetch_or(1ull << (dev & 63));
      }
      // Groups share no body, so every class runs concurrently: the big islands (one long block
      // each) on their own highest-priority side stream, launched first; the single-island buckets
      // (classes 10..15, few long blocks) one per side stream, largest first; the many short packed
      // groups on the tick's stream. Side streams fork from the tick's stream and join it after.
      const bool big = ng > g_small;
      auto lst = [&](int c) { return S.cls_list.p + (size_t)c * ng; };
      static_assert(PH_VEL_ISL5 - PH_VEL_ISL0 + 1 == ISLAND_BUCKETS, "a profile phase per island bucket");
      P.end(PH_VEL_PREP, st);
      if (big) {
        // every class's timer starts here, on the tick's stream, and stops on the class's own
        // stream: each reads as the time from the fork to that class's end
        P.begin(PH_VEL_BIG, st);
        for (int b = 0; b < ISLAND_BUCKETS; ++b)
          if (cls_n[10 + b]) P.begin(PH_VEL_ISL0 + b, st);
        RP_CUDA(cudaEventRecord(W.ev_fork_, st));
        for (int k = 0; k < WorldGpu::kAux; ++k) RP_CUDA(cudaStreamWaitEvent(W.aux_[k], W.ev_fork_, 0));
        cudaStream_t sg = W.aux_[WorldGpu::kAux - 1];
        // big islands: per-row inverse inertias for the staged stream, then one CTA each, per bucket
        uint32_t nbig = cls_n[20] + cls_n[21] + cls_n[22];
        if (nbig) {
          S.big_x.ensure(7 * (size_t)nsched + 7); S.big_j.ensure(nsched + 1);
          k_big_rows_x<<<nblk(nsched), T, 0, sg>>>(nsched, S.ord_main.p, S.row_isl2.p, S.g_class.p, R, B, SR, S.big_x.p,
                                                   S.big_j.p); RP_COUNT_LAUNCH(1);
        }
        for (int b = BIG_BUCKETS - 1; b >= 0; --b) {
          uint32_t n = cls_n[20 + b];
          if (!n) continue;
          if (b == BIG_BUCKETS - 1)
            k_vel_solve_big<128><<<n, 128, big_smem<128>(kBigBodies[b], kBigLevels[b]), sg>>>(
                kBigBodies[b], kBigLevels[b], 20u + (uint32_t)b, n, lst(20 + b), S.g_class.p, S.gb_start.p, S.gb_cnt.p,
                S.gb_list.p, SM, SR, S.big_x.p, S.big_j.p, B, W.warm_a.p, W.warm_b.p, S.acc_jn.p, S.acc_jt.p, iters, tol, stats,
                S.row_islid.p, S.isl_final.p);
          else
            k_vel_solve_big<64><<<n, 64, big_smem<64>(kBigBodies[b], kBigLevels[b]), sg>>>(
                kBigBodies[b], kBigLevels[b], 20u + (uint32_t)b, n, lst(20 + b), S.g_class.p, S.gb_start.p, S.gb_cnt.p,
                S.gb_list.p, SM, SR, S.big_x.p, S.big_j.p, B, W.warm_a.p, W.warm_b.p, S.acc_jn.p, S.acc_jt.p, iters, tol, stats,
                S.row_islid.p, S.isl_final.p);
          RP_COUNT_LAUNCH(1);
        }
        if (cls_n[2]) {  // islands beyond the big buckets: a warp each over global memory
          k_vel_solve<<<nblk(cls_n[2] * 32, 128), 128, 0, sg>>>(cls_n[2], nc, SM, R, B, S.acc_jn.p, S.acc_jt.p, S.wm_idx.p,
                                                                 W.warm_a.p, W.warm_b.p, iters, tol, stats, S.g_class.p,
                                                                 lst(2), S.row_islid.p, S.isl_final.p); RP_COUNT_LAUNCH(1);
        }
        P.end(PH_VEL_BIG, sg);
        for (int b = ISLAND_BUCKETS - 1; b >= 0; --b) {
          cudaStream_t sb = W.aux_[b];
          uint32_t n = cls_n[10 + b];
          if (!n) continue;
          OnchipLayout lay = onchip_layout(kIslandRows[b], kIslandBodies[b], 1u);
          auto kern = W.tuning_.island_threads == 32    ? k_vel_solve_onchip<false, 32>
                      : W.tuning_.island_threads == 64  ? k_vel_solve_onchip<false, 64>
                      : W.tuning_.island_threads == 256 ? k_vel_solve_onchip<false, 256>
                                                        : k_vel_solve_onchip<false, 128>;
          kern<<<n, W.tuning_.island_threads, lay.bytes, sb>>>(
              lay, 0u, n, lst(10 + b), 10u + (uint32_t)b, S.g_class.p, S.gb_start.p, S.gb_cnt.p, S.gb_list.p,
              S.g_nisl.p, SM, SR, B, W.warm_a.p, W.warm_b.p, S.acc_jn.p, S.acc_jt.p, iters, tol, stats, S.row_islid.p,
              S.isl_final.p); RP_COUNT_LAUNCH(1);
          P.end(PH_VEL_ISL0 + b, sb);
        }
      }
      P.begin(PH_VEL_PACKED, st);
      if (g_small > 0) {
        auto kern = W.tuning_.packed_threads == 32 ? k_vel_solve_onchip<true, 32>
                  : W.tuning_.packed_threads == 128 ? k_vel_solve_onchip<true, 128> : k_vel_solve_onchip<true, 64>;
        kern<<<g_small, W.tuning_.packed_threads, lay_packed.bytes, st>>>(
            lay_packed, 0u, g_small, nullptr, 3u, S.g_class.p, S.gb_start.p, S.gb_cnt.p, S.gb_list.p, S.g_nisl.p, SM, SR, B,
            W.warm_a.p, W.warm_b.p, S.acc_jn.p, S.acc_jt.p, iters, tol, stats, S.row_islid.p, S.isl_final.p);
        RP_COUNT_LAUNCH(1);
      }
      P.end(PH_VEL_PACKED, st);
      if (big) {
        for (int k = 0; k < WorldGpu::kAux; ++k) {
          RP_CUDA(cudaEventRecord(W.ev_join_[k], W.aux_[k]));
          RP_CUDA(cudaStreamWaitEvent(st, W.ev_join_[k], 0));
        }
      }
      // every solve island's last-sweep residual, written by its rows, binned once
      k_res_hist<<<nblk(nisl), T, 0, st>>>(nisl, S.isl_final.p, stats); RP_COUNT_LAUNCH(1);
    }
    P.end(PH_VEL_SOLVE, st);
    joints_store_warm(W, R, nc, S.acc_jn.p, st);
    if (W.feat_log_) {
      S.targets.ensure(3 * (size_t)nc + 3);
      k_row_targets<<<nblk(nc), T, 0, st>>>(nc, R, S.acc_jn.p, S.acc_jt.p, S.targets.p); RP_COUNT_LAUNCH(1);
    }
    P.begin(PH_WARM_CACHE, st);
    // ---- warm-start cache for the next tick (solver.rs:917-944)
    {
      S.woff.ensure(nc + 1); S.wpos.ensure(nc + 1);
      k_warm_new_flags<<<nblk(nc), T, 0, st>>>(nc, R, S.acc_jn.p, S.acc_jt.p, S.wpos.p); RP_COUNT_LAUNCH(1);
      uint32_t n_new = exclusive_scan_total(S, S.wpos.p, S.woff.p, nc, st);
      // new keys alone first (positions without the old-kept offsets), to test old entries against
      W.warm_key2.ensure(n_new + W.n_warm + 1); W.warm_a2.ensure(n_new + W.n_warm + 1); W.warm_b2.ensure(n_new + W.n_warm + 1);
      k_warm_new_write<<<nblk(nc), T, 0, st>>>(nc, R, S.acc_jn.p, S.acc_jt.p, S.wpos.p, S.woff.p, nullptr, nullptr, 0,
                                               W.warm_key2.p, W.warm_a2.p, W.warm_b2.p); RP_COUNT_LAUNCH(1);
      uint32_t n_kept = 0;
      S.wflag.ensure(W.n_warm + 1);
      DBuf<uint4>& kept_k = S.kept_k;
      DBuf<float4>& kept_a = S.kept_a;
      DBuf<float4>& kept_b = S.kept_b;
      if (W.n_warm > 0) {
        k_warm_old_flags<<<nblk(W.n_warm), T, 0, st>>>(W.n_warm, W.warm_key.p, W.warm_key2.p, n_new, W.alive_d.p, W.dyn.p,
                                                       W.awake.p, nb, S.wflag.p); RP_COUNT_LAUNCH(1);
        kept_k.ensure(W.n_warm + 1); kept_a.ensure(W.n_warm + 1); kept_b.ensure(W.n_warm + 1);
        size_t bytes = 0;
        S.counts.ensure(4);
        RP_CUDA(cub::DeviceSelect::Flagged(nullptr, bytes, W.warm_key.p, S.wflag.p, kept_k.p, S.counts.p + 3, W.n_warm, st));
        S.cub_tmp.ensure(bytes + 16);
        RP_CUDA(cub::DeviceSelect::Flagged(S.cub_tmp.p, bytes, W.warm_key.p, S.wflag.p, kept_k.p, S.counts.p + 3, W.n_warm, st));
        RP_COUNT_LAUNCH(2);
        RP_CUDA(cub::DeviceSelect::Flagged(S.cub_tmp.p, bytes, W.warm_a.p, S.wflag.p, kept_a.p, S.counts.p + 3, W.n_warm, st));
        RP_COUNT_LAUNCH(2);
        RP_CUDA(cub::DeviceSelect::Flagged(S.cub_tmp.p, bytes, W.warm_b.p, S.wflag.p, kept_b.p, S.counts.p + 3, W.n_warm, st));
        RP_COUNT_LAUNCH(2);
        RP_CUDA(cudaMemcpyAsync(&n_kept, S.counts.p + 3, 4, cudaMemcpyDeviceToHost, st));
        RP_CUDA(cudaStreamSynchronize(st));
      }
      if (n_kept == 0) {
        std::swap(W.warm_key.p, W.warm_key2.p); std::swap(W.warm_key.cap, W.warm_key2.cap);
        std::swap(W.warm_a.p, W.warm_a2.p); std::swap(W.warm_a.cap, W.warm_a2.cap);
        std::swap(W.warm_b.p, W.warm_b2.p); std::swap(W.warm_b.cap, W.warm_b2.cap);
        W.n_warm = n_new;
      } else {
        // merge: new entry k at off[k] + #kept below its key; kept entry j at j + #new below its key
        W.warm_key.ensure(n_new + n_kept + 1); W.warm_a.ensure(n_new + n_kept + 1); W.warm_b.ensure(n_new + n_kept + 1);
        k_warm_new_write<<<nblk(nc), T, 0, st>>>(nc, R, S.acc_jn.p, S.acc_jt.p, S.wpos.p, S.woff.p, nullptr, kept_k.p,
                                                 n_kept, W.warm_key.p, W.warm_a.p, W.warm_b.p); RP_COUNT_LAUNCH(1);
        k_warm_merge_kept<<<nblk(n_kept), T, 0, st>>>(n_kept, kept_k.p, kept_a.p, kept_b.p, W.warm_key2.p, n_new, W.warm_key.p,
                                        W.warm_a.p, W.warm_b.p); RP_COUNT_LAUNCH(1);
        W.n_warm = n_new + n_kept;
        RP_CUDA(cudaStreamSynchronize(st));
      }
    }
    P.end(PH_WARM_CACHE, st);
    P.begin(PH_VEL_SHOCK, st);
    // ---- shock propagation (solver.rs:964-993)
    if (ng > 0) {
      k_shock_keys<<<nblk(nsched), T, 0, st>>>(nsched, S.rows_sched.p, S.r_ab.p, S.r_flags.p, W.pos.p, ctx.up, S.key64.p); RP_COUNT_LAUNCH(1);
      sort_pairs_u64(S, S.key64.p, S.key64b.p, S.rows_sched.p, S.tmp32.p, nsched, 0, 64, st);  // by height key, stable
      k_gather_u32<<<nblk(nsched), T, 0, st>>>(nsched, S.tmp32.p, S.row_isl2.p, S.tmp32b.p); RP_COUNT_LAUNCH(1);     // their groups
      sort_pairs_u32(S, S.tmp32b.p, S.woff.p, S.tmp32.p, S.rows_sched2.p, nsched, 0, 32, st);   // by group, stable
      build_schedule(S, stats + STAT_ERR, nsched, ng, S.rows_sched2.p, S.g_start.p, S.g_cnt.p, S.ord_vs.p, S.lvl_off_vs,
                     S.lvl_start_vs, S.nlev_vs, nullptr, nullptr, st);
      Sched SV{S.ord_vs.p, S.lvl_off_vs.p, S.lvl_start_vs.p, S.nlev_vs.p};
      k_vel_shock<<<nblk(ng * 32, 128), 128, 0, st>>>(ng, SV, R, B, ctx.up, S.acc_jn.p); RP_COUNT_LAUNCH(1);
      // restitution for the contacts W6 leaves alone (jointed bodies); without joints there are none
      if (nj) { k_restitution<<<nblk(ng * 32, 128), 128, 0, st>>>(ng, nc, SM, R, B, S.acc_jn.p); RP_COUNT_LAUNCH(1); }
      // the W6 bounce passes (solver.rs:1009-1241); every kernel after the count returns at once
      // when no row bounces
      w6::W6V V6 = w6_view(S);
      w6::k_w6_count<<<nblk(nc), T, 0, st>>>(nc, R, S.acc_jn.p, V6, stats); RP_COUNT_LAUNCH(1);
      w6::k_w6_setup<<<1, w6::kBT, 0, st>>>(nc, nb, R, B, S.acc_jn.p, S.acc_jt.p, jointed, ctx.dt, V6); RP_COUNT_LAUNCH(1);
      w6::k_w6_solve<<<4, 64, 0, st>>>(R, B, S.acc_jn.p, jointed, V6, stats); RP_COUNT_LAUNCH(1);
      w6::k_w6_pseudo_setup<<<1, w6::kBT, 0, st>>>(nc, nb, R, B, S.acc_jn.p, S.acc_jt.p, jointed, V6); RP_COUNT_LAUNCH(1);
      w6::k_w6_pseudo_solve<<<4, 64, 0, st>>>(R, B, jointed, V6, stats); RP_COUNT_LAUNCH(1);
      w6::k_w6_pseudo_finish<<<nblk(nb), T, 0, st>>>(nb, V6); RP_COUNT_LAUNCH(1);
    }
    P.end(PH_VEL_SHOCK, st);
    k_after_solve<<<nblk(nc), T, 0, st>>>(nc, R, S.acc_jn.p, S.acc_jt.p, S.loaded.p, S.c_n.p, stats); RP_COUNT_LAUNCH(1);
  }
  // ---- stage 4
  P.begin(PH_BALLISTIC, st);
  if (nc > 0) { k_constrained<<<nblk(nc), T, 0, st>>>(nc, S.c_a.p, S.c_b.p, W.col_body.p, S.constrained.p); RP_COUNT_LAUNCH(1); }
  joints_mark_constrained(W, S.constrained.p, st);
  if (nb > 0) { k_ballistic_init<<<nblk(nb), T, 0, st>>>(nb, S.constrained.p, S.loaded.p, jointed, S.ballistic.p); RP_COUNT_LAUNCH(1); }
  Sched SM{S.ord_main.p, S.lvl_off.p, S.lvl_start.p, S.nlev.p};
  if (ctx.nisl > 0) {
    k_ballistic<<<nblk(ctx.nisl * 32, 128), 128, 0, st>>>(ctx.nisl, SM, R, B, S.c_pt.p, S.c_n.p, W.last_lin.p, ctx.dt,
                                                          S.ballistic.p); RP_COUNT_LAUNCH(1);
  }
  P.end(PH_BALLISTIC, st);
  P.begin(PH_INTEGRATE, st);
  if (nb > 0) {
    k_integrate<<<nblk(nb, 128), 128, 0, st>>>(nb, B, S.ballistic.p, W.last_lin.p, ctx.dt, S.orig_pos.p, S.orig_rot.p,
                                               S.pred_pos.p, S.pred_rot.p, S.w6_ctr.p, S.w6_pl.p, S.w6_pa.p);
    RP_COUNT_LAUNCH(1);
  }
  P.end(PH_INTEGRATE, st);
  // ---- stage 5: position pass (step.rs:284-309); its contacts are the scheduled rows
  if (ctx.nisl > 0) {
    P.begin(PH_POS_ITER, st);
    S.pc_lb.ensure(nc + 1);
    k_pos_anchors<<<nblk(nc), T, 0, st>>>(nc, R, S.c_pt.p, S.orig_pos.p, S.orig_rot.p, S.pc_lb.p); RP_COUNT_LAUNCH(1);
    if (nj) RP_CUDA(cudaMemsetAsync(W.jlam.p, 0, sizeof(float) * 6 * (size_t)nj, st));  // Joints::begin_step
    Sched SPP = npp ? Sched{S.ord_pp.p, S.lvl_off_pp.p, S.lvl_start_pp.p, S.nlev_pp.p} : SM;
    const uint32_t ngr = ctx.nisl;
    auto pos_launch = [&](auto tag, uint32_t n, const uint32_t* list, uint32_t skip) {
      constexpr int G = decltype(tag)::value;
      if (!n) return;
      uint32_t warps = (n + (32u / G) - 1) / (32u / G);
      k_pos_iterations<G><<<nblk(warps * 32, 128), 128, 0, st>>>(
          n, list, skip, S.g_class.p, nc, SPP, R, B, (int)W.iters_p_, 0, ctx.up, S.c_pt.p, S.c_n.p, S.pc_lb.p, S.split_l.p,
          S.split_a.p, W.joints_d.p, W.jlam.p, S.orig_pos.p, S.orig_rot.p, ctx.dt); RP_COUNT_LAUNCH(1);
    };
    if (npp) {
      // jointed islands of up to 128 / 256 rows (a ragdoll or two): 2 / 4 lanes each, the rest 8.
      // The pass is bound by the instructions a warp issues: more islands per warp put more of its
      // lanes to work per instruction (ragdolls: 2 / 4 / 8 lanes 21 ms, 4 / 8 / 32 lanes 27 ms,
      // 32 lanes for every island 58 ms; lane counts change no result bit)
      pos_launch(std::integral_constant<int, 2>{}, cls_n[10], S.cls_list.p + 10 * (size_t)ngr, 0u);
      pos_launch(std::integral_constant<int, 4>{}, cls_n[11], S.cls_list.p + 11 * (size_t)ngr, 0u);
      pos_launch(std::integral_constant<int, 8>{}, ngr, nullptr, (1u << 10) | (1u << 11));
    } else if (ngr) {
      // no joints: the groups the velocity solve keeps on chip run the pass on chip as well (the
      // single-island buckets on the side streams, the packed groups here); the big and
      // global-memory islands keep the warp kernel, on the big islands' side stream
      static std::atomic<unsigned long long> pos_attr{0};
      int dev = 0;
      RP_CUDA(cudaGetDevice(&dev));
      const PosLayout top = pos_layout(kIslandRows[ISLAND_BUCKETS - 1], kIslandBodies[ISLAND_BUCKETS - 1]);
      if (!((pos_attr.load() >> (dev & 63)) & 1ull)) {
        for (auto f : {k_pos_onchip<32>, k_pos_onchip<64>, k_pos_onchip<128>, k_pos_onchip<256>})
          RP_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)top.bytes));
        pos_attr.fetch_or(1ull << (dev & 63));
      }
      auto onchip = [&](uint32_t threads) {
        return threads == 32 ? k_pos_onchip<32> : threads == 64 ? k_pos_onchip<64>
             : threads == 128 ? k_pos_onchip<128> : k_pos_onchip<256>;
      };
      const uint32_t g_small = ctx.g_small;
      RP_CUDA(cudaEventRecord(W.ev_fork_, st));
      for (int k = 0; k < WorldGpu::kAux; ++k) RP_CUDA(cudaStreamWaitEvent(W.aux_[k], W.ev_fork_, 0));
      {
        cudaStream_t sg = W.aux_[WorldGpu::kAux - 1];
        const uint32_t skip = (1u << 3) | (0x3Fu << 10);  // classes run on chip
        const uint32_t warps = ngr;
        k_pos_iterations<32><<<nblk(warps * 32, 128), 128, 0, sg>>>(
            ngr, nullptr, skip, S.g_class.p, nc, SPP, R, B, (int)W.iters_p_, 0, ctx.up, S.c_pt.p, S.c_n.p, S.pc_lb.p,
            S.split_l.p, S.split_a.p, W.joints_d.p, W.jlam.p, S.orig_pos.p, S.orig_rot.p, ctx.dt); RP_COUNT_LAUNCH(1);
      }
      for (int b = ISLAND_BUCKETS - 1; b >= 0; --b) {
        const uint32_t n = cls_n[10 + b];
        if (!n) continue;
        const PosLayout lay = pos_layout(kIslandRows[b], kIslandBodies[b]);
        onchip(W.tuning_.island_threads)<<<n, W.tuning_.island_threads, lay.bytes, W.aux_[b]>>>(
            lay, n, S.cls_list.p + (size_t)(10 + b) * ngr, 10u + (uint32_t)b, S.g_class.p, S.gb_start.p, S.gb_cnt.p,
            S.gb_list.p, S.body_grp.p, S.body_local.p, SPP, R, B, (int)W.iters_p_, ctx.up, S.c_pt.p, S.c_n.p, S.pc_lb.p,
            S.split_l.p, S.split_a.p, stats); RP_COUNT_LAUNCH(1);
      }
      if (g_small) {
        const uint32_t gr = W.tuning_.group_rows;
        const PosLayout lay = pos_layout(WG_ROWS(gr), WG_BODIES(gr));
        onchip(W.tuning_.packed_threads)<<<g_small, W.tuning_.packed_threads, lay.bytes, st>>>(
            lay, g_small, nullptr, 3u, S.g_class.p, S.gb_start.p, S.gb_cnt.p, S.gb_list.p, S.body_grp.p, S.body_local.p,
            SPP, R, B, (int)W.iters_p_, ctx.up, S.c_pt.p, S.c_n.p, S.pc_lb.p, S.split_l.p, S.split_a.p, stats);
        RP_COUNT_LAUNCH(1);
      }
      for (int k = 0; k < WorldGpu::kAux; ++k) {
        RP_CUDA(cudaEventRecord(W.ev_join_[k], W.aux_[k]));
        RP_CUDA(cudaStreamWaitEvent(st, W.ev_join_[k], 0));
      }
    }
    P.end(PH_POS_ITER, st);
    P.begin(PH_POS_SHOCK, st);
    // shock projection in (height key, index) order at the poses the iterations left
    uint32_t nsched = ctx.nsched;
    k_shock_keys<<<nblk(nsched), T, 0, st>>>(nsched, S.rows_sched.p, S.r_ab.p, S.r_flags.p, W.pos.p, ctx.up, S.key64.p); RP_COUNT_LAUNCH(1);
    sort_pairs_u64(S, S.key64.p, S.key64b.p, S.rows_sched.p, S.tmp32.p, nsched, 0, 64, st);
    k_gather_u32<<<nblk(nsched), T, 0, st>>>(nsched, S.tmp32.p, S.row_isl2.p, S.tmp32b.p); RP_COUNT_LAUNCH(1);
    sort_pairs_u32(S, S.tmp32b.p, S.woff.p, S.tmp32.p, S.rows_sched2.p, nsched, 0, 32, st);
    build_schedule(S, stats + STAT_ERR, nsched, ctx.nisl, S.rows_sched2.p, S.g_start.p, S.g_cnt.p, S.ord_ps.p, S.lvl_off_ps,
                   S.lvl_start_ps, S.nlev_ps, nullptr, nullptr, st);
    Sched SP{S.ord_ps.p, S.lvl_off_ps.p, S.lvl_start_ps.p, S.nlev_ps.p};
    k_pos_iterations<32><<<nblk(ctx.nisl * 32, 128), 128, 0, st>>>(ctx.nisl, nullptr, 0u, S.g_class.p, nc, SP, R, B, 1, 1,
                                                                   ctx.up, S.c_pt.p, S.c_n.p, S.pc_lb.p, S.split_l.p,
                                                                   S.split_a.p, W.joints_d.p, W.jlam.p, S.orig_pos.p,
                                                                   S.orig_rot.p, ctx.dt); RP_COUNT_LAUNCH(1);
    P.end(PH_POS_SHOCK, st);
  }
  // ---- stages 6 and 7
  P.begin(PH_STAGE6, st);
  if (nc > 0) { k_touching<<<nblk(nc), T, 0, st>>>(nc, S.c_a.p, S.c_b.p, S.c_pt.p, W.col_body.p, S.touching.p); RP_COUNT_LAUNCH(1); }
  if (nb > 0) {
    k_stage6<<<nblk(nb), T, 0, st>>>(nb, B, S.orig_pos.p, S.pred_pos.p, S.pred_rot.p, S.split_l.p, S.split_a.p,
                                     S.touching.p, jointed, ctx.dt, W.last_lin.p, W.awake.p, W.sleep_ticks.p, W.sleep_allowed.p,
                                     stats); RP_COUNT_LAUNCH(1);
  }
  uint32_t ncap = W.capacity() > nb ? W.capacity() : nb;
  k_count_sleeping<<<nblk(ncap), T, 0, st>>>(ncap, W.awake.p, stats); RP_COUNT_LAUNCH(1);
  P.end(PH_STAGE6, st);
}

}  // namespace rp
