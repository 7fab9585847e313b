// joints.cu -- D6 joints in the tick: the joint records on the device, the joint parts of the
// island count (islands.rs:27-93), the joint velocity rows (solver.rs:644-664) written into the
// same row arrays as the contacts, their warm start and warm cache (solver.rs:699-712, 946-952),
// and the World-level joint API (world.rs:718-720, 966-968).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "joints.cuh"

namespace rp {

namespace {
const int T = 256;
inline int nblk(uint32_t n, int t = T) { return n ? (int)((n + t - 1) / t) : 1; }
}  // namespace

// ------------------------------------------------------------------ kernels
__global__ void k_joint_union(uint32_t nj, const JointGpu* __restrict__ J, const float* __restrict__ inv_mass,
                              uint32_t* uf) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nj) return;
  uint32_t a = J[j].a, b = J[j].b;
  if (inv_mass[a] > 0.0f && inv_mass[b] > 0.0f) uf_union(uf, a, b);
}
// route_to_island for joints (islands.rs:70-77)
__global__ void k_joint_marks(uint32_t nj, const JointGpu* __restrict__ J, const float* __restrict__ inv_mass,
                              uint32_t* uf, uint32_t* mark) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nj) return;
  uint32_t a = J[j].a, b = J[j].b;
  bool da = inv_mass[a] > 0.0f, db = inv_mass[b] > 0.0f;
  if (!da && !db) return;
  mark[uf_find(uf, da ? a : b)] = 1;
}
__global__ void k_joint_count(uint32_t nj, const JointGpu* __restrict__ J, BodiesV B, float dt, uint32_t* cnt) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nj) return;
  cnt[j] = joint_rows_dev(J[j], B, dt, [](const JRowD&, uint32_t) {});
}
// Rows of joint j at R[base + off[j] + k]. Warm start (solver.rs:703-712): the previous rows'
// impulses when the joint has an entry with the same row count and tags, each clamped to its
// row's bounds. A joint row stores: ra.w = 1 / k, t1 = (row count on the first row, index in the
// joint, gamma, target), t2.x = warm impulse, mu = (lam_min, lam_max, 0, tag), la.x = the joint's
// index (bits).
__global__ void k_joint_build(uint32_t nj, const JointGpu* __restrict__ J, BodiesV B, float dt,
                              const uint32_t* __restrict__ off, uint32_t base, RowsV R,
                              const uint32_t* __restrict__ jw_n, const uint8_t* __restrict__ jw_tag,
                              const float* __restrict__ jw_lam, float* acc_jn, float2* acc_jt, uint32_t* uf) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nj) return;
  const JointGpu& jt = J[j];
  const uint32_t r0 = base + off[j], wn = jw_n[j];
  bool tags_match = true, dyn_a = false, dyn_b = false;
  uint32_t n = joint_rows_dev(jt, B, dt, [&](const JRowD& r, uint32_t k) {
    uint32_t i = r0 + k;
    tags_match = tags_match && k < wn && jw_tag[JMAX_ROWS * (size_t)j + k] == (uint8_t)r.tag;
    if (k == 0) { dyn_a = r.wa > 0.0f; dyn_b = r.wb > 0.0f; }
    R.ab[i] = make_uint2(jt.a, jt.b);
    R.flags[i] = RF_JOINT | (r.angular ? RF_JANG : 0u) | (r.wa > 0.0f ? RF_WA : 0u) | (r.wb > 0.0f ? RF_WB : 0u) |
                 (k == 0 ? RF_JFIRST : 0u) | (r.legacy ? RF_JLEG : 0u) | (r.carrier ? RF_JNULL : 0u);
    R.inv[i] = make_float2(r.wa, r.wb);
    R.ra[i] = f4(r.ra, r.m_eff);
    R.rb[i] = f4(r.rb, r.inv_sum);
    R.n[i] = f4(r.u, 0.0f);
    // t1.x: the joint's row count on its first row (the unit's length, set below), t1.y: the row's
    // index, t1.w: the target (the bias of an original distance row)
    R.t1[i] = make_float4(0.0f, (float)k, r.gamma, r.legacy ? r.bias : r.target);
    R.t2[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    R.mu[i] = make_float4(r.lo, r.hi, 0.0f, __uint_as_float(r.tag));
    R.la[i] = make_float4(__uint_as_float(j), 0.0f, 0.0f, 0.0f);
    acc_jn[i] = 0.0f;
    acc_jt[i] = make_float2(0.0f, 0.0f);
  });
  if (n == 0) return;
  R.t1[r0].x = (float)n;
  // distance rows start cold (solver.rs:704-705); a carrier row is no row
  if (tags_match && wn == n && !(jt.flags & JF_DIST) && !(R.flags[r0] & RF_JNULL)) {
    for (uint32_t k = 0; k < n; ++k) {
      const uint32_t i = r0 + k;
      const float4 mu = R.mu[i];
      R.flags[i] |= RF_JWARM;
      R.t2[i].x = clampf(jw_lam[JMAX_ROWS * (size_t)j + k], mu.x, mu.y);
    }
  }
  // the joint's rows join its two bodies' solve island when both can move
  if (dyn_a && dyn_b) uf_union(uf, jt.a, jt.b);
}
__global__ void k_joint_roots(uint32_t njr, uint32_t base, RowsV R, uint32_t* uf, uint32_t* row_root) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= njr) return;
  uint32_t r = base + i;
  uint2 ab = R.ab[r];
  row_root[r] = uf_find(uf, (R.flags[r] & RF_WA) ? ab.x : ab.y);
}
// Joints solved this tick replace their cache entry; the others keep theirs (solver.rs:946-952).
__global__ void k_joint_store(uint32_t nj, const JointGpu* __restrict__ J, const uint32_t* __restrict__ cnt,
                              const uint32_t* __restrict__ off,
                              uint32_t base, RowsV R, const float* __restrict__ acc_jn, uint32_t* jw_n,
                              uint8_t* jw_tag, float* jw_lam) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nj) return;
  uint32_t n = cnt[j];
  // distance rows are not kept (solver.rs:945-947); a carrier row is no row
  if (n == 0 || (J[j].flags & JF_DIST) || (R.flags[base + off[j]] & RF_JNULL)) return;
  jw_n[j] = n;
  for (uint32_t k = 0; k < n; ++k) {
    uint32_t r = base + off[j] + k;
    jw_tag[JMAX_ROWS * (size_t)j + k] = (uint8_t)__float_as_uint(R.mu[r].w);
    jw_lam[JMAX_ROWS * (size_t)j + k] = acc_jn[r];
  }
}
__global__ void k_joint_constrained(uint32_t nj, const JointGpu* __restrict__ J, uint8_t* constrained) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nj) return;
  constrained[J[j].a] = 1;
  constrained[J[j].b] = 1;
}
// Cache entries of joints touching `body` dropped (mode 0), or of joints with a removed body (mode 1).
__global__ void k_joint_warm_filter(uint32_t nj, const JointGpu* __restrict__ J, int mode, uint32_t body,
                                    const uint8_t* __restrict__ alive, uint32_t* jw_n) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nj) return;
  uint32_t a = J[j].a, b = J[j].b;
  bool drop = mode == 0 ? (a == body || b == body) : !(alive[a] && alive[b]);
  if (drop) jw_n[j] = 0xFFFFFFFFu;
}

// ------------------------------------------------------------------ host launchers
void joints_ref_islands(WorldGpu& W, uint32_t* uf, uint32_t* root_mark, bool unions, cudaStream_t st) {
  uint32_t nj = W.num_joints();
  if (!nj) return;
  if (unions) k_joint_union<<<nblk(nj), T, 0, st>>>(nj, W.joints_d.p, W.inv_mass.p, uf);
  else k_joint_marks<<<nblk(nj), T, 0, st>>>(nj, W.joints_d.p, W.inv_mass.p, uf, root_mark);
  RP_COUNT_LAUNCH(1);
}
uint32_t joints_count_rows(WorldGpu& W, float dt, const BodiesV& B, cudaStream_t st) {
  uint32_t nj = W.num_joints();
  W.njr_ = 0;
  if (!nj) return 0;
  W.jr_cnt.ensure(nj + 1); W.jr_off.ensure(nj + 1);
  k_joint_count<<<nblk(nj, 128), 128, 0, st>>>(nj, W.joints_d.p, B, dt, W.jr_cnt.p); RP_COUNT_LAUNCH(1);
  W.njr_ = exclusive_scan_total(*W.s_, W.jr_cnt.p, W.jr_off.p, nj, st);
  return W.njr_;
}
void joints_build_rows(WorldGpu& W, float dt, const BodiesV& B, const RowsV& R, uint32_t base, float* acc_jn,
                       float2* acc_jt, uint32_t* uf, cudaStream_t st) {
  uint32_t nj = W.num_joints();
  if (!nj || !W.njr_) return;
  k_joint_build<<<nblk(nj, 128), 128, 0, st>>>(nj, W.joints_d.p, B, dt, W.jr_off.p, base, R, W.jw_n.p, W.jw_tag.p,
                                               W.jw_lam.p, acc_jn, acc_jt, uf); RP_COUNT_LAUNCH(1);
}
void joints_row_roots(WorldGpu& W, const RowsV& R, uint32_t base, uint32_t njr, uint32_t* uf, uint32_t* row_root,
                      cudaStream_t st) {
  if (!njr) return;
  k_joint_roots<<<nblk(njr), T, 0, st>>>(njr, base, R, uf, row_root); RP_COUNT_LAUNCH(1);
}
void joints_store_warm(WorldGpu& W, const RowsV& R, uint32_t base, const float* acc_jn, cudaStream_t st) {
  uint32_t nj = W.num_joints();
  if (!nj || !W.njr_) return;
  k_joint_store<<<nblk(nj), T, 0, st>>>(nj, W.joints_d.p, W.jr_cnt.p, W.jr_off.p, base, R, acc_jn, W.jw_n.p, W.jw_tag.p, W.jw_lam.p);
  RP_COUNT_LAUNCH(1);
}
void joints_mark_constrained(WorldGpu& W, uint8_t* constrained, cudaStream_t st) {
  uint32_t nj = W.num_joints();
  if (!nj) return;
  k_joint_constrained<<<nblk(nj), T, 0, st>>>(nj, W.joints_d.p, constrained); RP_COUNT_LAUNCH(1);
}

// ------------------------------------------------------------------ WorldGpu: joint API
// The batch world body `b` belongs to (bodies before the first world count as world 0).
uint32_t WorldGpu::world_of(uint32_t b) const {
  auto it = std::upper_bound(h_wb_start_.begin(), h_wb_start_.end(), b);
  return it == h_wb_start_.begin() ? 0u : (uint32_t)(it - h_wb_start_.begin()) - 1u;
}
// Joints::add_ball / add_hinge (bodies.rs:326-338); kind 2: a D6 joint with every axis locked
uint32_t WorldGpu::add_joint(uint32_t kind, uint32_t a, uint32_t b, const float fa[7], const float fb[7], uint32_t axis) {
  JointHost j{};
  j.a = a; j.b = b;
  for (int k = 0; k < 7; ++k) { j.fa[k] = fa[k]; j.fb[k] = fb[k]; }
  for (int k = 0; k < 3; ++k) { j.en[k] = true; j.en[3 + k] = kind == 2 || (kind == 1 && (uint32_t)k != axis); }
  j.hinge = kind == 1 ? (int)axis : -1;
  if (batch_ && !h_wb_start_.empty()) {
    uint32_t wa = world_of(a), wb = world_of(b);
    if (wa != wb) throw std::invalid_argument("a joint in a batch joins two bodies of one world");
    if (!h_joints_.empty() && wa < world_of(h_joints_.back().a))
      throw std::invalid_argument("a batch's joints are added in world order");
  }
  h_joints_.push_back(j);
  joints_dirty_ = true;
  return (uint32_t)h_joints_.size() - 1;
}
// Joints::add_distance_joint_at + set_distance_damping (bodies.rs:273-305): rest and anchors made
// finite, compliance and damping finite and >= 0.
uint32_t WorldGpu::add_distance_joint(uint32_t a, uint32_t b, const float la[3], const float lb[3], float rest,
                                      float compliance, float damping) {
  JointHost j{};
  j.a = a; j.b = b;
  j.kind = 1;
  j.hinge = -1;
  auto fin0 = [](float x) { return std::isfinite(x) ? x : 0.0f; };
  for (int k = 0; k < 3; ++k) { j.fa[k] = fin0(la[k]); j.fb[k] = fin0(lb[k]); }
  j.fa[6] = 1.0f; j.fb[6] = 1.0f;
  j.rest = fin0(rest);
  j.dcomp = std::max(fin0(compliance), 0.0f);
  j.ddamp = std::max(fin0(damping), 0.0f);
  if (batch_ && !h_wb_start_.empty()) {
    uint32_t wa = world_of(a), wb = world_of(b);
    if (wa != wb) throw std::invalid_argument("a joint in a batch joins two bodies of one world");
    if (!h_joints_.empty() && wa < world_of(h_joints_.back().a))
      throw std::invalid_argument("a batch's joints are added in world order");
  }
  h_joints_.push_back(j);
  joints_dirty_ = true;
  return (uint32_t)h_joints_.size() - 1;
}
// leave_hinge (bodies.rs:876-878): limiting or driving another rotational axis drops the stored
// hinge axis
static void leave_hinge(WorldGpu::JointHost& j, bool angular, uint32_t axis) {
  if (angular && j.hinge >= 0 && j.hinge != (int)axis) j.hinge = -1;
}
// Joints::set_d6_limit_t / set_d6_limit_r (bodies.rs:367-391)
void WorldGpu::set_joint_limit(uint32_t id, bool angular, uint32_t axis, bool on, float lo, float hi) {
  JointHost& j = h_joints_.at(id);
  uint32_t ax = (angular ? 3u : 0u) + axis;
  j.lim[ax] = on;
  j.lo[ax] = lo; j.hi[ax] = hi;
  if (on) {
    j.en[ax] = true;
    leave_hinge(j, angular, axis);
  }
  joints_dirty_ = true;
}
// An axis locked (enabled) or free, and its XPBD compliance (0: rigid).
void WorldGpu::set_joint_axis(uint32_t id, bool angular, uint32_t axis, bool enabled, float compliance) {
  JointHost& j = h_joints_.at(id);
  uint32_t ax = (angular ? 3u : 0u) + axis;
  j.en[ax] = enabled;
  j.comp[ax] = compliance;
  joints_dirty_ = true;
}
// Joints::set_d6_drive_t / set_d6_drive_r (bodies.rs:354-366)
void WorldGpu::set_joint_drive(uint32_t id, bool angular, uint32_t axis, bool on, float target, float kp, float kd,
                               float max_impulse, bool vel_mode) {
  JointHost& j = h_joints_.at(id);
  uint32_t ax = (angular ? 3u : 0u) + axis;
  j.drive[ax] = on;
  j.dtarget[ax] = target; j.dkp[ax] = kp; j.dkd[ax] = kd; j.dmax[ax] = max_impulse; j.vel[ax] = vel_mode;
  if (on) {
    j.en[ax] = true;
    leave_hinge(j, angular, axis);
  }
  joints_dirty_ = true;
}
// Joints::set_d6_damping (bodies.rs:376-383): negative or non-finite values become 0
void WorldGpu::set_joint_damping(uint32_t id, bool angular, uint32_t axis, float damping, float friction) {
  JointHost& j = h_joints_.at(id);
  uint32_t ax = (angular ? 3u : 0u) + axis;
  auto clean = [](float x) { return std::isfinite(x) && x > 0.0f ? x : 0.0f; };
  j.damp[ax] = clean(damping);
  j.fric[ax] = clean(friction);
  joints_dirty_ = true;
}
// d6_hinge_axis (bodies.rs:891-901): the stored hinge axis; else the one free rotational axis
// (neither locked, limited nor driven); else a compliant rotational axis at least 100x softer than
// the other two.
static int hinge_of(const WorldGpu::JointHost& j) {
  if (j.hinge >= 0) return j.hinge < 3 ? j.hinge : -1;
  int free_axis = -1, n = 0;
  for (int i = 0; i < 3; ++i)
    if (!(j.en[3 + i] && !j.lim[3 + i] && !j.drive[3 + i])) { free_axis = i; n++; }
  if (n == 1) return free_axis;
  auto c = [&](int i) {
    float x = j.comp[3 + i];
    return j.en[3 + i] && std::isfinite(x) && x > 0.0f ? x : 0.0f;
  };
  for (int i = 0; i < 3; ++i) {
    if (!(j.en[3 + i] && c(i) > 0.0f)) continue;
    bool all = true;
    for (int k = 0; k < 3; ++k) all = all && (k == i || c(i) >= 100.0f * c(k));
    if (all) return i;
  }
  return -1;
}
template <class T>
static void grow_keep(DBuf<T>& d, size_t old_n, size_t new_n, cudaStream_t st) {
  if (new_n <= d.cap) return;
  DBuf<T> nd;
  nd.ensure(new_n);
  if (old_n) RP_CUDA(cudaMemcpyAsync(nd.p, d.p, sizeof(T) * old_n, cudaMemcpyDeviceToDevice, st));
  RP_CUDA(cudaStreamSynchronize(st));
  std::swap(d.p, nd.p);
  std::swap(d.cap, nd.cap);
}
void WorldGpu::upload_joints() {
  if (!joints_dirty_) return;
  const uint32_t nj = num_joints();
    std::vector<JointGpu> h(nj ? nj : 1);
  std::vector<uint8_t> jointed(cap_b_ > nb_ ? cap_b_ : (nb_ ? nb_ : 1), 0);
  std::vector<unsigned long long> keys;
  for (uint32_t i = 0; i < nj; ++i) {
    const JointHost& s = h_joints_[i];
    JointGpu& g = h[i];
    std::memset(&g, 0, sizeof(g));
    g.a = s.a; g.b = s.b;
    uint32_t f = 0;
    bool rdrive = false;
    for (int k = 0; k < 6; ++k) {
      if (s.en[k]) f |= 1u << k;
      if (s.lim[k]) f |= 1u << (JF_LIMIT_SHIFT + k);
      if (s.drive[k]) f |= 1u << (JF_DRIVE_SHIFT + k);
      if (s.vel[k]) f |= 1u << (JF_VEL_SHIFT + k);
      g.lo[k] = s.lo[k]; g.hi[k] = s.hi[k];
      g.comp[k] = s.comp[k]; g.damp[k] = s.damp[k]; g.fric[k] = s.fric[k];
      g.dtarget[k] = s.dtarget[k]; g.dmax[k] = s.dmax[k];
      if (k >= 3 && s.drive[k] && s.vel[k]) rdrive = true;
      if (s.drive[k] || s.comp[k] > 0.0f) f |= JF_FULL;
    }
    if (s.kind == 1) {  // a distance joint: rest lo[0], compliance comp[0], damping damp[0]
      f = JF_DIST;
      const bool anchored = !(s.fa[0] == 0.0f && s.fa[1] == 0.0f && s.fa[2] == 0.0f) ||
                            !(s.fb[0] == 0.0f && s.fb[1] == 0.0f && s.fb[2] == 0.0f) || s.ddamp > 0.0f;
      if (anchored) f |= JF_ANCH;
      for (int k = 0; k < 6; ++k) { g.lo[k] = 0.0f; g.hi[k] = 0.0f; g.comp[k] = 0.0f; g.damp[k] = 0.0f; }
      g.lo[0] = s.rest; g.comp[0] = s.dcomp; g.damp[0] = s.ddamp;
      rdrive = false;
    } else {
      f |= (uint32_t)(hinge_of(s) + 1) << JF_HINGE_SHIFT;
    }
    g.flags = f;
    g.fa_p = make_float4(s.fa[0], s.fa[1], s.fa[2], 0.0f); g.fa_q = make_float4(s.fa[3], s.fa[4], s.fa[5], s.fa[6]);
    g.fb_p = make_float4(s.fb[0], s.fb[1], s.fb[2], 0.0f); g.fb_q = make_float4(s.fb[3], s.fb[4], s.fb[5], s.fb[6]);
    // bit 0: in a joint; bit 1: in a joint with a rotational velocity drive (the motor overwrite)
    const uint8_t mark = rdrive ? 3 : 1;
    jointed[s.a] |= mark;
    jointed[s.b] |= mark;
    keys.push_back(s.a < s.b ? (((unsigned long long)s.a << 32) | s.b) : (((unsigned long long)s.b << 32) | s.a));
  }
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  // the cache keeps the entries of the joints it had; new joints start with none
  uint32_t had = (uint32_t)(jw_n.cap && jw_init_ ? jw_init_ : 0);
  grow_keep(jw_n, had, nj + 1, stream_);
  grow_keep(jw_tag, (size_t)JMAX_ROWS * had, (size_t)JMAX_ROWS * (nj + 1), stream_);
  grow_keep(jw_lam, (size_t)JMAX_ROWS * had, (size_t)JMAX_ROWS * (nj + 1), stream_);
  if (nj > had) RP_CUDA(cudaMemsetAsync(jw_n.p + had, 0xFF, 4 * (size_t)(nj - had), stream_));
  jw_init_ = nj;
  joints_d.ensure(nj + 1);
  jointed_d.ensure(jointed.size());
  jpair_keys.ensure(keys.size() + 1);
  jlam.ensure(6 * (size_t)nj + 6);
  if (nj) RP_CUDA(cudaMemcpyAsync(joints_d.p, h.data(), sizeof(JointGpu) * nj, cudaMemcpyHostToDevice, stream_));
  RP_CUDA(cudaMemcpyAsync(jointed_d.p, jointed.data(), jointed.size(), cudaMemcpyHostToDevice, stream_));
  if (!keys.empty())
    RP_CUDA(cudaMemcpyAsync(jpair_keys.p, keys.data(), 8 * keys.size(), cudaMemcpyHostToDevice, stream_));
  n_jpairs = (uint32_t)keys.size();
  RP_CUDA(cudaStreamSynchronize(stream_));
  joints_dirty_ = false;
}
void WorldGpu::drop_joint_warm_of(uint32_t body) {
  upload_joints();
  uint32_t nj = num_joints();
  if (!nj) return;
  k_joint_warm_filter<<<nblk(nj), T, 0, stream_>>>(nj, joints_d.p, 0, body, alive_d.p, jw_n.p); RP_COUNT_LAUNCH(1);
}
void WorldGpu::filter_joint_warm_alive() {
  upload_joints();
  uint32_t nj = num_joints();
  if (!nj) return;
  k_joint_warm_filter<<<nblk(nj), T, 0, stream_>>>(nj, joints_d.p, 1, 0u, alive_d.p, jw_n.p); RP_COUNT_LAUNCH(1);
}

}  // namespace rp
