// world_gpu.cu -- WorldGpu: the device-resident world (body state, colliders, warm-start cache,
// heightfield) and the host orchestration of the tick. Body-management calls mirror
// riftphys-world/src/world/world.rs; every state change happens on the world's stream.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "step_internal.cuh"

namespace rp {

// ------------------------------------------------------------------ materials and mass
// props() core table (riftphys-materials/src/materials.rs:97-110), MaterialId ordinals 0..13.
static const float kMat[14][4] = {
    {0.60f, 0.50f, 0.10f, 0.08f}, {0.05f, 0.03f, 0.02f, 0.02f}, {1.10f, 0.95f, 0.80f, 0.15f},
    {0.70f, 0.55f, 0.50f, 0.05f}, {1.30f, 1.05f, 0.00f, 0.12f}, {0.55f, 0.45f, 0.08f, 0.10f},
    {0.80f, 0.70f, 0.00f, 0.10f}, {0.90f, 0.80f, 0.00f, 0.12f}, {0.80f, 0.60f, 0.20f, 0.10f},
    {0.55f, 0.45f, 0.10f, 0.06f}, {1.10f, 0.95f, 0.00f, 0.18f}, {0.40f, 0.30f, 0.65f, 0.04f},
    {0.90f, 0.60f, 0.35f, 0.06f}, {0.61f, 0.47f, 0.40f, 0.05f}};
bool material_known(uint32_t id) { return id < 14; }
// mix_pair (geometric-mean friction, max restitution, 1e-6 quantised) and the curated overrides
// (materials.rs:250-305)
PairPropsHost table_pair_props(uint32_t a, uint32_t b) {
  const float* pa = kMat[a];
  const float* pb = kMat[b];
  PairPropsHost r;
  r.mu_s = quantize_mat(sqrtf(fabsf(pa[0] * pb[0])));
  r.mu_k = quantize_mat(sqrtf(fabsf(pa[1] * pb[1])));
  r.restitution = quantize_mat(rmax(pa[2], pb[2]));
  r.stribeck_v = quantize_mat(0.5f * (pa[3] + pb[3]));
  r.stiffness = 0.0f;
  uint32_t x = a < b ? a : b, y = a < b ? b : a;
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
    r.mu_s = quantize_mat(ov[0]); r.mu_k = quantize_mat(ov[1]);
    r.restitution = quantize_mat(ov[2]); r.stribeck_v = quantize_mat(ov[3]);
  }
  return r;
}
static bool valid_pos(float x) { return isfinite(x) && x > 0.0f; }
static bool finalize_mass(float m, float ix, float iy, float iz, float* im, float in[3]) {
  if (!valid_pos(m) || m < 1.0e-12f || !(valid_pos(ix) && valid_pos(iy) && valid_pos(iz))) {
    *im = 0; in[0] = in[1] = in[2] = 0; return false;
  }
  *im = 1.0f / m; in[0] = ix; in[1] = iy; in[2] = iz;
  return true;
}
// MassProps::from_{sphere,box,capsule}_density (riftphys-geom/src/mass.rs:75-145)
bool mass_from_density(uint32_t shape, const float d[3], float rho, float* im, float in[3]) {
  const float kPi = 3.14159265358979323846f, k43 = 4.0f / 3.0f, k112 = 1.0f / 12.0f;
  *im = 0; in[0] = in[1] = in[2] = 0;
  if (shape == SH_SPHERE) {
    float r = fabsf(d[0]);
    if (!(valid_pos(r) && valid_pos(rho))) return false;
    float r2 = r * r;
    float m = rho * (((k43 * kPi) * r2) * r);
    float ii = (0.4f * m) * r2;
    return finalize_mass(m, ii, ii, ii, im, in);
  }
  if (shape == SH_BOX) {
    float hx = fabsf(d[0]), hy = fabsf(d[1]), hz = fabsf(d[2]);
    if (!(isfinite(hx) && isfinite(hy) && isfinite(hz) && valid_pos(rho))) return false;
    float dx = hx * 2.0f, dy = hy * 2.0f, dz = hz * 2.0f;
    if (!(valid_pos(dx) && valid_pos(dy) && valid_pos(dz))) return false;
    float m = rho * ((dx * dy) * dz);
    float x2 = dx * dx, y2 = dy * dy, z2 = dz * dz;
    return finalize_mass(m, (k112 * m) * (y2 + z2), (k112 * m) * (x2 + z2), (k112 * m) * (x2 + y2), im, in);
  }
  if (shape == SH_CAPSULE) {
    float r = fabsf(d[0]), hh = fabsf(d[1]);
    if (!(valid_pos(r) && isfinite(rho) && rho > 0.0f)) return false;
    float h = hh * 2.0f, r2 = r * r;
    float m = rho * (((kPi * r2) * h) + (((k43 * kPi) * r2) * r));
    float ix = ((0.25f * m) * r2) + (((k112 * m) * h) * h);
    return finalize_mass(m, ix, (0.5f * m) * r2, ix, im, in);
  }
  return false;
}

// ------------------------------------------------------------------ small device kernels
__global__ void k_set_body(uint32_t i, float4 p, float4 q, float4 l, float4 a, float im, m3 ii, uint8_t dyn,
                           uint8_t sleep_ok, float4* pos, float4* rot, float4* lin, float4* ang, float4* last,
                           float* inv_mass, float* inv_I, uint8_t* d_dyn, uint8_t* awake, uint8_t* sa,
                           uint16_t* ticks, uint8_t* alive, float4 last_v) {
  pos[i] = p; rot[i] = q; lin[i] = l; ang[i] = a; last[i] = last_v;
  inv_mass[i] = im;
  float* o = inv_I + 9 * (size_t)i;
  o[0] = ii.c0.x; o[1] = ii.c0.y; o[2] = ii.c0.z; o[3] = ii.c1.x; o[4] = ii.c1.y; o[5] = ii.c1.z;
  o[6] = ii.c2.x; o[7] = ii.c2.y; o[8] = ii.c2.z;
  d_dyn[i] = dyn; awake[i] = 1; ticks[i] = 0; sa[i] = sleep_ok; alive[i] = 1;
}
// Bodies::set_pose (dynamics.rs:130-134) + World::set_body_vel (world.rs:674-676) helpers
__global__ void k_set_pose(uint32_t i, float4 p, float4 q, float4* pos, float4* rot) {
  f3 pp = xyz(p);
  q4 qq = asq(q);
  if (vfin(pp)) pos[i] = f4(fin_v(pp), pos[i].w);
  if (qfin(qq)) rot[i] = f4q(fin_q(qq));
}
__global__ void k_set_vel(uint32_t i, float4 l, float4 a, float4* lin, float4* ang, float4* last) {
  f3 ll = xyz(l), aa = xyz(a);
  if (vfin(ll)) lin[i] = f4(fin_v(ll));
  if (vfin(aa)) ang[i] = f4(fin_v(aa));
  last[i] = f4(ll);
}
// World::apply_impulse (world.rs:689-692): wake, then Bodies::apply_impulse
__global__ void k_apply_impulse(uint32_t i, float4 j, float4* lin, const float* inv_mass, uint8_t* awake, uint16_t* ticks) {
  awake[i] = 1; ticks[i] = 0;
  float im = inv_mass[i];
  f3 jj = xyz(j);
  if (im > 0.0f && vfin(jj)) lin[i] = f4(fin_v(xyz(lin[i]) + jj * im));
}
// Bodies::deactivate (dynamics.rs:213-220)
__global__ void k_deactivate(uint32_t i, float4* lin, float4* ang, float* inv_mass, float* inv_I, uint8_t* dyn, uint8_t* alive) {
  lin[i] = make_float4(0, 0, 0, 0); ang[i] = make_float4(0, 0, 0, 0);
  inv_mass[i] = 0.0f; dyn[i] = 0; alive[i] = 0;
  for (int k = 0; k < 9; ++k) inv_I[9 * (size_t)i + k] = 0.0f;
}
// Warm-cache filters: mode 0 drops keys holding `body` (World::drop_warm_of, world.rs:818-826);
// mode 1 keeps keys whose bodies are alive or terrain (restore_carried_state, world.rs:946-950).
__global__ void k_warm_filter(uint32_t n, const uint4* __restrict__ k, int mode, uint32_t body,
                              const uint8_t* __restrict__ alive, uint32_t nb, uint8_t* keep) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  uint4 x = k[e];
  bool kp;
  if (mode == 0) kp = x.x != body && x.y != body;
  else {
    auto al = [&](uint32_t b) { return b == 0xFFFFFFFFu || (b < nb && alive[b] != 0); };
    kp = al(x.x) && al(x.y);
  }
  keep[e] = kp ? 1 : 0;
}
// Snapshot restore of the bodies still alive (lib.rs:1771-1785): set_body_pose / set_body_vel,
// then the carried last velocities and sleep state (world.rs:937-945).
__global__ void k_restore_bodies(uint32_t n, const float4* __restrict__ sp, const float4* __restrict__ sr,
                                 const float4* __restrict__ sl, const float4* __restrict__ sa,
                                 const float4* __restrict__ slast, const uint8_t* __restrict__ alive, float4* pos,
                                 float4* rot, float4* lin, float4* ang, float4* last) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (alive[i]) {
    f3 p = xyz(sp[i]); q4 q = asq(sr[i]);
    if (vfin(p)) pos[i] = f4(fin_v(p), pos[i].w);
    if (qfin(q)) rot[i] = f4q(fin_q(q));
    f3 l = xyz(sl[i]), a = xyz(sa[i]);
    if (vfin(l)) lin[i] = f4(fin_v(l));
    if (vfin(a)) ang[i] = f4(fin_v(a));
    last[i] = f4(l);
  }
  last[i] = slast[i];
}

// ------------------------------------------------------------------ WorldGpu
WorldGpu::WorldGpu(uint32_t max_bodies, uint32_t max_colliders) : cap_b_(max_bodies), cap_c_(max_colliders) {
  RP_CUDA(cudaGetDevice(&dev_));
  RP_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  // the side streams carry the long single-island solves: highest priority, so the block
  // scheduler places them before the many short packed groups queued on the main stream
  int prio_least = 0, prio_greatest = 0;
  RP_CUDA(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
  for (int k = 0; k < kAux; ++k) {
    RP_CUDA(cudaStreamCreateWithPriority(&aux_[k], cudaStreamNonBlocking, prio_greatest));
    RP_CUDA(cudaEventCreateWithFlags(&ev_join_[k], cudaEventDisableTiming));
  }
  RP_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
  {
    // the stream-ordered pool keeps what a tick frees, so regrowing scratch never returns memory
    // to the driver mid-run (this process's default pool on this device only)
    int dev = 0;
    cudaMemPool_t pool;
    RP_CUDA(cudaGetDevice(&dev));
    RP_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t thr = UINT64_MAX;
    RP_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  }
  s_ = new Scratch();
  size_t cb = cap_b_ > 0 ? cap_b_ : 1, cc = cap_c_ > 0 ? cap_c_ : 1;
  pos.ensure(cb); rot.ensure(cb); lin.ensure(cb); ang.ensure(cb); last_lin.ensure(cb);
  inv_mass.ensure(cb); inv_I.ensure(9 * cb);
  dyn.ensure(cb); awake.ensure(cb); sleep_allowed.ensure(cb); alive_d.ensure(cb); sleep_ticks.ensure(cb);
  col_body.ensure(cc); col_kind.ensure(cc); col_mat.ensure(cc); col_dims.ensure(cc);
  pair_table.ensure(14 * 14 * 5);
  d_stats.ensure(STAT_COUNT);
  // SleepManager::new(capacity): every slot awake, 0 ticks, sleep allowed (sleep.rs:15-27)
  RP_CUDA(cudaMemsetAsync(awake.p, 1, cb, stream_));
  RP_CUDA(cudaMemsetAsync(sleep_ticks.p, 0, cb * 2, stream_));
  RP_CUDA(cudaMemsetAsync(sleep_allowed.p, 1, cb, stream_));
  RP_CUDA(cudaMemsetAsync(alive_d.p, 0, cb, stream_));
  RP_CUDA(cudaMemsetAsync(d_stats.p, 0, STAT_COUNT * 4, stream_));
  upload_pair_table();
  RP_CUDA(cudaStreamSynchronize(stream_));
}
WorldGpu::~WorldGpu() {
  cudaStreamSynchronize(stream_);
  for (int k = 0; k < kAux; ++k) cudaStreamSynchronize(aux_[k]);
  delete s_;
  for (int k = 0; k < kAux; ++k) { cudaEventDestroy(ev_join_[k]); cudaStreamDestroy(aux_[k]); }
  cudaEventDestroy(ev_fork_);
  cudaStreamDestroy(stream_);
}

void WorldGpu::upload_pair_table() {
  std::vector<float> t(14 * 14 * 5);
  for (uint32_t a = 0; a < 14; ++a)
    for (uint32_t b = 0; b < 14; ++b) {
      std::pair<uint32_t, uint32_t> key = a <= b ? std::make_pair(a, b) : std::make_pair(b, a);
      PairPropsHost p = table_pair_props(a, b);
      for (auto& o : overrides_) if (o.first == key) p = o.second;  // World::pair_props (world.rs:982-986)
      float* q = &t[5 * (a * 14 + b)];
      q[0] = p.mu_s; q[1] = p.mu_k; q[2] = p.restitution; q[3] = p.stribeck_v; q[4] = p.stiffness;
    }
  RP_CUDA(cudaMemcpyAsync(pair_table.p, t.data(), t.size() * 4, cudaMemcpyHostToDevice, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
}
void WorldGpu::set_pair_props(uint32_t a, uint32_t b, const PairPropsHost& p) {
  std::pair<uint32_t, uint32_t> key = a <= b ? std::make_pair(a, b) : std::make_pair(b, a);
  overrides_.erase(std::remove_if(overrides_.begin(), overrides_.end(), [&](auto& o) { return o.first == key; }),
                   overrides_.end());
  overrides_.push_back({key, p});
  upload_pair_table();
}

// World::add_body (world.rs:595-614), Bodies::add (dynamics.rs:98-117), add_collider (:616-622)
static void body_init(const float pose[7], const float vel[6], float inv_mass_in, const float inertia[3], bool dynamic,
                      float4* P, float4* Q, float4* L, float4* A, float* im, m3* ii, uint8_t* is_dyn, float4* last) {
  f3 p = mk3(pose[0], pose[1], pose[2]);
  q4 q = mkq(pose[3], pose[4], pose[5], pose[6]);
  f3 l = mk3(vel[0], vel[1], vel[2]), a = mk3(vel[3], vel[4], vel[5]);
  float im_arg = dynamic ? inv_mass_in : 0.0f;
  m3 inertia_m = mdiag(mk3(inertia[0], inertia[1], inertia[2]));
  float det = mdet(inertia_m);
  bool has_inv = dynamic && isfinite(det) && det > 0.0f;
  m3 inv_local = has_inv ? minverse(inertia_m) : mzero();
  bool d = dynamic && isfinite(im_arg) && im_arg > 0.0f;
  float imv = d ? fin0(im_arg) : 0.0f;
  bool inv_fin = vfin(inv_local.c0) && vfin(inv_local.c1) && vfin(inv_local.c2);
  *ii = !d ? mzero() : (has_inv && inv_fin ? inv_local : mdiag(splat(imv)));
  *P = f4(vfin(p) ? p : mk3(0, 0, 0));
  *Q = f4q(fin_q(q));
  *L = f4(vfin(l) ? l : mk3(0, 0, 0));
  *A = f4(vfin(a) ? a : mk3(0, 0, 0));
  *im = imv;
  *is_dyn = d ? 1 : 0;
  *last = f4(l);
}
uint32_t WorldGpu::add_body(const float pose[7], const float vel[6], uint32_t shape, const float dims[3], float im_in,
                            const float inertia[3], bool dynamic, uint32_t mat, bool sleep_ok) {
  float4 P, Q, L, A, last; float im; m3 ii; uint8_t d;
  body_init(pose, vel, im_in, inertia, dynamic, &P, &Q, &L, &A, &im, &ii, &d, &last);
  uint32_t id = nb_++;
  k_set_body<<<1, 1, 0, stream_>>>(id, P, Q, L, A, im, ii, d, sleep_ok ? 1 : 0, pos.p, rot.p, lin.p, ang.p, last_lin.p,
                                   inv_mass.p, inv_I.p, dyn.p, awake.p, sleep_allowed.p, sleep_ticks.p, alive_d.p, last); RP_COUNT_LAUNCH(1);
  h_alive_.push_back(1);
  uint32_t c = ncol_++;
  if (batch_) worlds_dirty_ = true;
  h_col_body_.push_back(id); h_col_kind_.push_back(shape); h_col_mat_.push_back(mat);
  float dd[4] = {dims[0], shape == SH_SPHERE ? 0.0f : dims[1], shape == SH_BOX ? dims[2] : 0.0f, 0.0f};
  h_col_dims_.insert(h_col_dims_.end(), dd, dd + 4);
  RP_CUDA(cudaMemcpyAsync(col_body.p + c, &h_col_body_[c], 4, cudaMemcpyHostToDevice, stream_));
  RP_CUDA(cudaMemcpyAsync(col_kind.p + c, &h_col_kind_[c], 4, cudaMemcpyHostToDevice, stream_));
  RP_CUDA(cudaMemcpyAsync(col_mat.p + c, &h_col_mat_[c], 4, cudaMemcpyHostToDevice, stream_));
  RP_CUDA(cudaMemcpyAsync(col_dims.p + c, &h_col_dims_[4 * c], 16, cudaMemcpyHostToDevice, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
  return id;
}
void WorldGpu::add_bodies_bulk(uint32_t n, const float* pose7, const float* vel6, const uint32_t* shape, const float* dims3,
                               const float* im_in, const float* inertia3, const uint8_t* dynamic, const uint32_t* mat,
                               const uint8_t* sleep_ok) {
  if (n == 0) return;
  std::vector<float4> P(n), Q(n), L(n), A(n), last(n), dims(n);
  std::vector<float> im(n), ii(9 * (size_t)n);
  std::vector<uint8_t> d(n), ones(n, 1), sa(n);
  std::vector<uint16_t> zeros(n, 0);
  std::vector<uint32_t> cb(n);
  for (uint32_t k = 0; k < n; ++k) {
    m3 m; uint8_t dd;
    body_init(pose7 + 7 * (size_t)k, vel6 + 6 * (size_t)k, im_in[k], inertia3 + 3 * (size_t)k, dynamic[k] != 0, &P[k],
              &Q[k], &L[k], &A[k], &im[k], &m, &dd, &last[k]);
    d[k] = dd;
    float* o = &ii[9 * (size_t)k];
    o[0] = m.c0.x; o[1] = m.c0.y; o[2] = m.c0.z; o[3] = m.c1.x; o[4] = m.c1.y; o[5] = m.c1.z;
    o[6] = m.c2.x; o[7] = m.c2.y; o[8] = m.c2.z;
    sa[k] = sleep_ok[k];
    cb[k] = nb_ + k;
    const float* dm = dims3 + 3 * (size_t)k;
    dims[k] = make_float4(dm[0], shape[k] == SH_SPHERE ? 0.0f : dm[1], shape[k] == SH_BOX ? dm[2] : 0.0f, 0.0f);
  }
  uint32_t b0 = nb_, c0 = ncol_;
  auto up = [&](void* dst, const void* src, size_t bytes) {
    RP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream_));
  };
  up(pos.p + b0, P.data(), 16 * (size_t)n); up(rot.p + b0, Q.data(), 16 * (size_t)n);
  up(lin.p + b0, L.data(), 16 * (size_t)n); up(ang.p + b0, A.data(), 16 * (size_t)n);
  up(last_lin.p + b0, last.data(), 16 * (size_t)n); up(inv_mass.p + b0, im.data(), 4 * (size_t)n);
  up(inv_I.p + 9 * (size_t)b0, ii.data(), 36 * (size_t)n); up(dyn.p + b0, d.data(), n);
  up(awake.p + b0, ones.data(), n); up(sleep_ticks.p + b0, zeros.data(), 2 * (size_t)n);
  up(sleep_allowed.p + b0, sa.data(), n); up(alive_d.p + b0, ones.data(), n);
  up(col_body.p + c0, cb.data(), 4 * (size_t)n); up(col_kind.p + c0, shape, 4 * (size_t)n);
  up(col_mat.p + c0, mat, 4 * (size_t)n); up(col_dims.p + c0, dims.data(), 16 * (size_t)n);
  RP_CUDA(cudaStreamSynchronize(stream_));
  for (uint32_t k = 0; k < n; ++k) {
    h_alive_.push_back(1);
    h_col_body_.push_back(b0 + k); h_col_kind_.push_back(shape[k]); h_col_mat_.push_back(mat[k]);
    h_col_dims_.push_back(dims[k].x); h_col_dims_.push_back(dims[k].y); h_col_dims_.push_back(dims[k].z);
    h_col_dims_.push_back(0.0f);
  }
  nb_ += n;
  ncol_ += n;
  if (batch_) worlds_dirty_ = true;
}

// The last tick's feature rows (24 floats) and converged impulses (3 floats) of the contacts that
// had a movable body, in contact order (the learned warm start's training data).
void WorldGpu::get_row_features(std::vector<float>& feats, std::vector<float>& targets) {
  feats.clear(); targets.clear();
  uint32_t n = n_contacts;
  if (!feat_log_ || !n || s_->feat.cap < 24 * (size_t)n || s_->targets.cap < 3 * (size_t)n) return;
  std::vector<float> f(24 * (size_t)n), t(3 * (size_t)n);
  std::vector<uint8_t> v(n);
  RP_CUDA(cudaMemcpyAsync(f.data(), s_->feat.p, 4 * f.size(), cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaMemcpyAsync(t.data(), s_->targets.p, 4 * t.size(), cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaMemcpyAsync(v.data(), s_->feat_valid.p, n, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
  for (uint32_t k = 0; k < n; ++k) {
    if (!v[k]) continue;
    feats.insert(feats.end(), f.begin() + 24 * (size_t)k, f.begin() + 24 * (size_t)(k + 1));
    targets.insert(targets.end(), t.begin() + 3 * (size_t)k, t.begin() + 3 * (size_t)(k + 1));
  }
}
// The predictions the last tick's warm start was offered, per contact in contact order:
// (normal, friction 1, friction 2, 1) or zeros where none was (no model, no movable body, or an
// island solved over global memory).
void WorldGpu::get_row_predictions(std::vector<float>& pred4) {
  uint32_t n = n_contacts;
  pred4.assign(4 * (size_t)n, 0.0f);
  if (!pred_valid_ || !n) return;
  RP_CUDA(cudaMemcpyAsync(pred4.data(), s_->pred_used.p, 16 * (size_t)n, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
}

void WorldGpu::begin_world() {
  if (!h_players_.empty()) throw std::invalid_argument("a world with players cannot become a batch");
  batch_ = true;
  h_wb_start_.push_back(nb_);
  h_wc_start_.push_back(ncol_);
  worlds_dirty_ = true;
}
void WorldGpu::upload_worlds() {
  if (!batch_ || !worlds_dirty_) return;
  uint32_t nw = num_worlds();
  std::vector<uint32_t> cw(ncol_ ? ncol_ : 1, 0), ws(nw + 1);
  for (uint32_t w = 0; w < nw; ++w) {
    uint32_t c0 = h_wc_start_[w], c1 = w + 1 < nw ? h_wc_start_[w + 1] : ncol_;
    for (uint32_t c = c0; c < c1; ++c) cw[c] = w;
    ws[w] = c0;
  }
  ws[nw] = ncol_;
  col_world.ensure(cw.size());
  world_col_start.ensure(nw + 1);
  RP_CUDA(cudaMemcpyAsync(col_world.p, cw.data(), 4 * cw.size(), cudaMemcpyHostToDevice, stream_));
  RP_CUDA(cudaMemcpyAsync(world_col_start.p, ws.data(), 4 * ws.size(), cudaMemcpyHostToDevice, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
  worlds_dirty_ = false;
}

void WorldGpu::filter_warm(int mode, uint32_t body) {
  if (n_warm == 0) return;
  const int T = 256;
  Scratch& S = *s_;
  S.wflag.ensure(n_warm + 1);
  k_warm_filter<<<(n_warm + T - 1) / T, T, 0, stream_>>>(n_warm, warm_key.p, mode, body, alive_d.p, nb_, S.wflag.p); RP_COUNT_LAUNCH(1);
  warm_key2.ensure(n_warm + 1); warm_a2.ensure(n_warm + 1); warm_b2.ensure(n_warm + 1);
  S.counts.ensure(4);
  size_t bytes = 0;
  RP_CUDA(cub::DeviceSelect::Flagged(nullptr, bytes, warm_key.p, S.wflag.p, warm_key2.p, S.counts.p, n_warm, stream_));
  S.cub_tmp.ensure(bytes + 16);
  RP_CUDA(cub::DeviceSelect::Flagged(S.cub_tmp.p, bytes, warm_key.p, S.wflag.p, warm_key2.p, S.counts.p, n_warm, stream_));
  RP_COUNT_LAUNCH(2);
  RP_CUDA(cub::DeviceSelect::Flagged(S.cub_tmp.p, bytes, warm_a.p, S.wflag.p, warm_a2.p, S.counts.p, n_warm, stream_));
  RP_COUNT_LAUNCH(2);
  RP_CUDA(cub::DeviceSelect::Flagged(S.cub_tmp.p, bytes, warm_b.p, S.wflag.p, warm_b2.p, S.counts.p, n_warm, stream_));
  RP_COUNT_LAUNCH(2);
  uint32_t n = 0;
  RP_CUDA(cudaMemcpyAsync(&n, S.counts.p, 4, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
  std::swap(warm_key.p, warm_key2.p); std::swap(warm_key.cap, warm_key2.cap);
  std::swap(warm_a.p, warm_a2.p); std::swap(warm_a.cap, warm_a2.cap);
  std::swap(warm_b.p, warm_b2.p); std::swap(warm_b.cap, warm_b2.cap);
  n_warm = n;
}
void WorldGpu::drop_warm_of(uint32_t b) { filter_warm(0, b); }

bool WorldGpu::remove_body(uint32_t id) {  // World::remove_body (world.rs:696-713)
  if (id >= nb_ || !h_alive_[id]) return false;
  h_alive_[id] = 0;
  k_deactivate<<<1, 1, 0, stream_>>>(id, lin.p, ang.p, inv_mass.p, inv_I.p, dyn.p, alive_d.p); RP_COUNT_LAUNCH(1);
  // colliders.retain(|c| c.body != id): later colliders shift down by one
  std::vector<uint32_t> keep;
  for (uint32_t c = 0; c < ncol_; ++c) if (h_col_body_[c] != id) keep.push_back(c);
  if (keep.size() != ncol_) {
    std::vector<uint32_t> b, k, m; std::vector<float> d;
    for (uint32_t c : keep) {
      b.push_back(h_col_body_[c]); k.push_back(h_col_kind_[c]); m.push_back(h_col_mat_[c]);
      d.insert(d.end(), &h_col_dims_[4 * c], &h_col_dims_[4 * c] + 4);
    }
    h_col_body_.swap(b); h_col_kind_.swap(k); h_col_mat_.swap(m); h_col_dims_.swap(d);
    ncol_ = (uint32_t)keep.size();
    if (ncol_) {
      RP_CUDA(cudaMemcpyAsync(col_body.p, h_col_body_.data(), 4 * (size_t)ncol_, cudaMemcpyHostToDevice, stream_));
      RP_CUDA(cudaMemcpyAsync(col_kind.p, h_col_kind_.data(), 4 * (size_t)ncol_, cudaMemcpyHostToDevice, stream_));
      RP_CUDA(cudaMemcpyAsync(col_mat.p, h_col_mat_.data(), 4 * (size_t)ncol_, cudaMemcpyHostToDevice, stream_));
      RP_CUDA(cudaMemcpyAsync(col_dims.p, h_col_dims_.data(), 16 * (size_t)ncol_, cudaMemcpyHostToDevice, stream_));
    }
  }
  drop_warm_of(id);
  drop_joint_warm_of(id);
  RP_CUDA(cudaStreamSynchronize(stream_));
  return true;
}
void WorldGpu::set_body_pose(uint32_t id, const float p[7]) {  // world.rs:501-513
  drop_warm_of(id);
  drop_joint_warm_of(id);
  k_set_pose<<<1, 1, 0, stream_>>>(id, make_float4(p[0], p[1], p[2], 0), make_float4(p[3], p[4], p[5], p[6]), pos.p, rot.p); RP_COUNT_LAUNCH(1);
  RP_CUDA(cudaStreamSynchronize(stream_));
}
void WorldGpu::set_body_vel(uint32_t id, const float v[6]) {
  k_set_vel<<<1, 1, 0, stream_>>>(id, make_float4(v[0], v[1], v[2], 0), make_float4(v[3], v[4], v[5], 0), lin.p, ang.p,
                                  last_lin.p); RP_COUNT_LAUNCH(1);
  RP_CUDA(cudaStreamSynchronize(stream_));
}
void WorldGpu::apply_impulse(uint32_t id, const float j[3]) {
  k_apply_impulse<<<1, 1, 0, stream_>>>(id, make_float4(j[0], j[1], j[2], 0), lin.p, inv_mass.p, awake.p, sleep_ticks.p); RP_COUNT_LAUNCH(1);
  RP_CUDA(cudaStreamSynchronize(stream_));
}
void WorldGpu::get_body_pose(uint32_t id, float out[7]) {
  float4 p, q;
  RP_CUDA(cudaMemcpyAsync(&p, pos.p + id, 16, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaMemcpyAsync(&q, rot.p + id, 16, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
  out[0] = p.x; out[1] = p.y; out[2] = p.z; out[3] = q.x; out[4] = q.y; out[5] = q.z; out[6] = q.w;
}
void WorldGpu::get_body_vel(uint32_t id, float out[6]) {
  float4 l, a;
  RP_CUDA(cudaMemcpyAsync(&l, lin.p + id, 16, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaMemcpyAsync(&a, ang.p + id, 16, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
  out[0] = l.x; out[1] = l.y; out[2] = l.z; out[3] = a.x; out[4] = a.y; out[5] = a.z;
}
void WorldGpu::get_body_states(uint32_t first, uint32_t count, float* out) {
  if (count == 0) return;
  std::vector<float4> p(count), q(count), l(count), a(count);
  RP_CUDA(cudaMemcpyAsync(p.data(), pos.p + first, 16 * (size_t)count, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaMemcpyAsync(q.data(), rot.p + first, 16 * (size_t)count, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaMemcpyAsync(l.data(), lin.p + first, 16 * (size_t)count, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaMemcpyAsync(a.data(), ang.p + first, 16 * (size_t)count, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
  for (uint32_t k = 0; k < count; ++k) {
    float* o = out + 13 * (size_t)k;
    o[0] = p[k].x; o[1] = p[k].y; o[2] = p[k].z; o[3] = q[k].x; o[4] = q[k].y; o[5] = q[k].z; o[6] = q[k].w;
    o[7] = l[k].x; o[8] = l[k].y; o[9] = l[k].z; o[10] = a[k].x; o[11] = a[k].y; o[12] = a[k].z;
  }
}
void WorldGpu::set_heightfield(uint32_t nx, uint32_t nz, float sx, float sz, float ox, float oz,
                               const std::vector<float>& h, float mn, float mx, uint32_t mat) {
  hf_h_.ensure(h.size() + 1);
  RP_CUDA(cudaMemcpyAsync(hf_h_.p, h.data(), 4 * h.size(), cudaMemcpyHostToDevice, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
  has_hf_ = true; hf_nx_ = nx; hf_nz_ = nz; hf_sx_ = sx; hf_sz_ = sz; hf_ox_ = ox; hf_oz_ = oz;
  hf_min_ = mn; hf_max_ = mx; hf_mat_ = mat;
}
void WorldGpu::clear_heightfield() { has_hf_ = false; }

// ------------------------------------------------------------------ the tick
void WorldGpu::step(float dt) {
  upload_worlds();
  upload_joints();
  AllocStreamScope alloc_scope(stream_);
  tick_ += 1;
  RP_CUDA(cudaMemsetAsync(d_stats.p, 0, STAT_COUNT * 4, stream_));
  run_players(dt);  // step.rs:51
  StepCtx ctx;
  ctx.dt = dt;
  ctx.g = mk3(q6(gravity_.x), q6(gravity_.y), q6(gravity_.z));
  ctx.up = len2(gravity_) > 0.0f ? -normalize(gravity_) : mk3(0, 1, 0);
  if (has_hf_) ctx.hf = HFView{hf_h_.p, hf_nx_, hf_nz_, hf_sx_, hf_sz_, hf_ox_, hf_oz_, hf_min_, hf_max_};
  ctx.hf_mat = hf_mat_;
  s_->pre_lin.ensure(nb_ + 1); s_->pre_ang.ensure(nb_ + 1);
  run_front(*this, ctx);
  run_solve(*this, ctx);
  st_.pairs = ctx.np;
  st_.contacts = ctx.nc;
  st_.islands = ctx.nref_isl;
  st_.rows_scheduled = ctx.nsched;
  stats_dirty_ = true;
  if (s_->prof.on) {
    RP_CUDA(cudaStreamSynchronize(stream_));
    s_->prof.collect();
  }
}
void WorldGpu::profile_enable(bool on) {
  s_->prof.on = on;
  s_->prof.reset();
}
int WorldGpu::profile_read(double* ms, uint64_t* calls, int cap) {
  int n = PH_COUNT < cap ? PH_COUNT : cap;
  for (int p = 0; p < n; ++p) { ms[p] = s_->prof.ms[p]; calls[p] = s_->prof.calls[p]; }
  return PH_COUNT;
}
const char* WorldGpu::phase_name(int p) { return (p >= 0 && p < PH_COUNT) ? kPhaseNames[p] : nullptr; }
void WorldGpu::synchronize() {
  RP_CUDA(cudaStreamSynchronize(stream_));
  RP_CUDA(cudaGetLastError());
}
const StepStatsHost& WorldGpu::stats() {
  if (stats_dirty_) {
    uint32_t h[STAT_COUNT];
    RP_CUDA(cudaMemcpyAsync(h, d_stats.p, STAT_COUNT * 4, cudaMemcpyDeviceToHost, stream_));
    RP_CUDA(cudaStreamSynchronize(stream_));
    st_.error_flags = h[STAT_ERR];
    st_.warm_matched = h[STAT_WARM_MATCHED];
    st_.bounce_rows = h[STAT_BOUNCE];
    st_.sweeps = h[STAT_SWEEPS];
    float r; std::memcpy(&r, &h[STAT_RESID], 4); st_.residual = r;
    st_.sleeping = h[STAT_SLEEPING];
    st_.levels = h[STAT_LEVELS];
    st_.max_batch = h[STAT_MAXBATCH];
    st_.row_sweeps = h[STAT_ROWSWEEPS];
    st_.groups_shared = h[STAT_GROUPS_SHARED];
    st_.groups_global = h[STAT_GROUPS_GLOBAL];
    st_.max_group_rows = h[STAT_MAX_GROUP_ROWS];
    st_.max_group_bodies = h[STAT_MAX_GROUP_BODIES];
    st_.islands_capped = h[STAT_ISLANDS_CAPPED];
    st_.pred_used = h[STAT_PRED_USED];
    st_.rows_capped = h[STAT_ROWS_CAPPED];
    for (int k = 0; k < 6; ++k) st_.res_hist[k] = h[STAT_RES_HIST + k];
    stats_dirty_ = false;
  }
  st_.warm_entries = n_warm;
  return st_;
}
void WorldGpu::get_pairs(std::vector<uint64_t>& out) {
  out.resize(n_pairs);
  if (n_pairs)
    RP_CUDA(cudaMemcpyAsync(out.data(), s_->pairs.p, 8 * (size_t)n_pairs, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
}
void WorldGpu::get_contacts(std::vector<ContactOut>& out) {
  uint32_t n = n_contacts;
  out.resize(n);
  if (!n) return;
  std::vector<uint32_t> a(n), b(n), lv(n, 0xFFFFFFFFu);
  std::vector<float4> p(n), nn(n);
  RP_CUDA(cudaMemcpyAsync(a.data(), s_->c_a.p, 4 * (size_t)n, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaMemcpyAsync(b.data(), s_->c_b.p, 4 * (size_t)n, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaMemcpyAsync(p.data(), s_->c_pt.p, 16 * (size_t)n, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaMemcpyAsync(nn.data(), s_->c_n.p, 16 * (size_t)n, cudaMemcpyDeviceToHost, stream_));
  if (levels_valid_) RP_CUDA(cudaMemcpyAsync(lv.data(), s_->row_level.p, 4 * (size_t)n, cudaMemcpyDeviceToHost, stream_));
  RP_CUDA(cudaStreamSynchronize(stream_));
  for (uint32_t k = 0; k < n; ++k) {
    ContactOut& c = out[k];
    c.a = a[k]; c.b = b[k];
    c.p[0] = p[k].x; c.p[1] = p[k].y; c.p[2] = p[k].z; c.depth = p[k].w;
    c.n[0] = nn[k].x; c.n[1] = nn[k].y; c.n[2] = nn[k].z; c.impulse = nn[k].w;
    c.level = lv[k];
  }
}

// ------------------------------------------------------------------ state blob
// Layout (little-endian): header of 48 bytes (magic "RPS1", version 1, tick, epoch, rng as u64,
// bodies, capacity, warm entries, joints as u32); per body 16 f32 (pos xyz, rot xyzw, lin xyz,
// ang xyz, last linear velocity xyz); per body its alive byte; per capacity slot the awake byte,
// then the sleep counter as u16; per warm entry its key (4 x u32) and la xyz, jn, jt xyz (7 f32);
// per joint its cached row count (u32, 0xFFFFFFFF: none), 32 row tags (u8) and 32 impulses (f32).
static constexpr uint32_t kStateMagic = 0x31535052u;  // "RPS1"
static constexpr uint64_t kStateHead = 48, kStateBody = 64, kStateWarm = 44, kStateJoint = 4 + 32 + 128;
static_assert(kJointRows == 32, "state blob: 32 cached rows per joint");
uint64_t WorldGpu::state_bytes() {
  uint64_t cap = cap_b_ > nb_ ? cap_b_ : nb_;
  return kStateHead + (kStateBody + 1) * nb_ + 3 * cap + kStateWarm * n_warm + kStateJoint * (uint64_t)num_joints();
}
void WorldGpu::state_export(uint8_t* out) {
  upload_joints();
  const uint32_t cap = cap_b_ > nb_ ? cap_b_ : nb_, nj = num_joints();
  std::vector<float4> hp(nb_), hr(nb_), hl(nb_), ha(nb_), hll(nb_);
  std::vector<uint8_t> aw(cap);
  std::vector<uint16_t> tk(cap);
  std::vector<uint4> wk(n_warm);
  std::vector<float4> wa(n_warm), wb(n_warm);
  std::vector<uint32_t> jn(nj);
  std::vector<uint8_t> jt((size_t)kJointRows * nj);
  std::vector<float> jl((size_t)kJointRows * nj);
  auto get = [&](void* d, const void* s, size_t b) { if (b) RP_CUDA(cudaMemcpyAsync(d, s, b, cudaMemcpyDeviceToHost, stream_)); };
  get(hp.data(), pos.p, 16ull * nb_); get(hr.data(), rot.p, 16ull * nb_); get(hl.data(), lin.p, 16ull * nb_);
  get(ha.data(), ang.p, 16ull * nb_); get(hll.data(), last_lin.p, 16ull * nb_);
  get(aw.data(), awake.p, cap); get(tk.data(), sleep_ticks.p, 2ull * cap);
  get(wk.data(), warm_key.p, 16ull * n_warm); get(wa.data(), warm_a.p, 16ull * n_warm); get(wb.data(), warm_b.p, 16ull * n_warm);
  if (nj) {
    get(jn.data(), jw_n.p, 4ull * nj);
    get(jt.data(), jw_tag.p, (size_t)kJointRows * nj);
    get(jl.data(), jw_lam.p, 4ull * kJointRows * nj);
  }
  RP_CUDA(cudaStreamSynchronize(stream_));
  uint8_t* p = out;
  auto put = [&](const void* v, size_t b) { std::memcpy(p, v, b); p += b; };
  const uint32_t hdr[2] = {kStateMagic, 1u};
  put(hdr, 8); put(&tick_, 8); put(&epoch_, 8); put(&rng_, 8);
  const uint32_t cnt[4] = {nb_, cap, n_warm, nj};
  put(cnt, 16);
  for (uint32_t i = 0; i < nb_; ++i) {
    const float v[16] = {hp[i].x, hp[i].y, hp[i].z, hr[i].x, hr[i].y, hr[i].z, hr[i].w, hl[i].x,
                         hl[i].y, hl[i].z, ha[i].x, ha[i].y, ha[i].z, hll[i].x, hll[i].y, hll[i].z};
    put(v, 64);
  }
  put(h_alive_.data(), nb_);
  put(aw.data(), cap);
  put(tk.data(), 2ull * cap);
  for (uint32_t e = 0; e < n_warm; ++e) {
    put(&wk[e], 16);
    const float v[7] = {wa[e].x, wa[e].y, wa[e].z, wa[e].w, wb[e].x, wb[e].y, wb[e].z};
    put(v, 28);
  }
  for (uint32_t j = 0; j < nj; ++j) {
    put(&jn[j], 4);
    put(&jt[(size_t)kJointRows * j], kJointRows);
    put(&jl[(size_t)kJointRows * j], 4 * kJointRows);
  }
}
void WorldGpu::state_import(const uint8_t* in, uint64_t bytes) {
  if (bytes < kStateHead) throw std::invalid_argument("state blob shorter than its header");
  uint32_t hdr[2];
  std::memcpy(hdr, in, 8);
  if (hdr[0] != kStateMagic || hdr[1] != 1u) throw std::invalid_argument("not a version 1 state blob");
  uint64_t tick, epoch, rng;
  std::memcpy(&tick, in + 8, 8); std::memcpy(&epoch, in + 16, 8); std::memcpy(&rng, in + 24, 8);
  uint32_t cnt[4];
  std::memcpy(cnt, in + 32, 16);
  const uint32_t cap = cap_b_ > nb_ ? cap_b_ : nb_;
  upload_joints();
  const uint32_t nj = num_joints(), nw = cnt[2];
  if (cnt[0] != nb_ || cnt[1] != cap || cnt[3] != nj)
    throw std::invalid_argument("state blob of another world: bodies " + std::to_string(cnt[0]) + ", capacity " +
                                std::to_string(cnt[1]) + ", joints " + std::to_string(cnt[3]) + "; this world has " +
                                std::to_string(nb_) + ", " + std::to_string(cap) + ", " + std::to_string(nj));
  const uint64_t need = kStateHead + (kStateBody + 1) * (uint64_t)nb_ + 3ull * cap + kStateWarm * (uint64_t)nw +
                        kStateJoint * (uint64_t)nj;
  if (bytes != need) throw std::invalid_argument("state blob size does not match its counts");
  if (!h_players_.empty()) throw std::invalid_argument("a world with players takes no state blob");
  const uint8_t* p = in + kStateHead;
  std::vector<float4> hp(nb_), hr(nb_), hl(nb_), ha(nb_), hll(nb_);
  for (uint32_t i = 0; i < nb_; ++i, p += 64) {
    float v[16];
    std::memcpy(v, p, 64);
    hp[i] = make_float4(v[0], v[1], v[2], 0.0f); hr[i] = make_float4(v[3], v[4], v[5], v[6]);
    hl[i] = make_float4(v[7], v[8], v[9], 0.0f); ha[i] = make_float4(v[10], v[11], v[12], 0.0f);
    hll[i] = make_float4(v[13], v[14], v[15], 0.0f);
  }
  if (std::memcmp(p, h_alive_.data(), nb_) != 0) throw std::invalid_argument("state blob's live bodies differ from this world's");
  p += nb_;
  const uint8_t* aw = p; p += cap;
  const uint8_t* tk = p; p += 2ull * cap;
  std::vector<uint4> wk(nw);
  std::vector<float4> wa(nw), wb(nw);
  for (uint32_t e = 0; e < nw; ++e, p += 44) {
    std::memcpy(&wk[e], p, 16);
    float v[7];
    std::memcpy(v, p + 16, 28);
    wa[e] = make_float4(v[0], v[1], v[2], v[3]);
    wb[e] = make_float4(v[4], v[5], v[6], 0.0f);
  }
  std::vector<uint32_t> jn(nj);
  std::vector<uint8_t> jt((size_t)kJointRows * nj);
  std::vector<float> jl((size_t)kJointRows * nj);
  for (uint32_t j = 0; j < nj; ++j) {
    std::memcpy(&jn[j], p, 4);
    std::memcpy(&jt[(size_t)kJointRows * j], p + 4, kJointRows);
    std::memcpy(&jl[(size_t)kJointRows * j], p + 4 + kJointRows, 4 * kJointRows);
    p += kStateJoint;
  }
  // the w lanes the device keeps (a body's pos.w / lin.w / ang.w) are untouched by the tick's
  // arithmetic and zero in every world; the blob restores the rest
  tick_ = tick; epoch_ = epoch; rng_ = rng;
  warm_key.ensure(nw + 1); warm_a.ensure(nw + 1); warm_b.ensure(nw + 1);
  auto put = [&](void* d, const void* s, size_t b) { if (b) RP_CUDA(cudaMemcpyAsync(d, s, b, cudaMemcpyHostToDevice, stream_)); };
  put(pos.p, hp.data(), 16ull * nb_); put(rot.p, hr.data(), 16ull * nb_); put(lin.p, hl.data(), 16ull * nb_);
  put(ang.p, ha.data(), 16ull * nb_); put(last_lin.p, hll.data(), 16ull * nb_);
  put(awake.p, aw, cap); put(sleep_ticks.p, tk, 2ull * cap);
  put(warm_key.p, wk.data(), 16ull * nw); put(warm_a.p, wa.data(), 16ull * nw); put(warm_b.p, wb.data(), 16ull * nw);
  n_warm = nw;
  if (nj) {
    put(jw_n.p, jn.data(), 4ull * nj);
    put(jw_tag.p, jt.data(), (size_t)kJointRows * nj);
    put(jw_lam.p, jl.data(), 4ull * kJointRows * nj);
  }
  RP_CUDA(cudaStreamSynchronize(stream_));
  stats_dirty_ = true;
}

// ------------------------------------------------------------------ rollback
SnapshotGpu* WorldGpu::snapshot_create() {  // lib.rs:1707-1752 + carried_state (world.rs:912-923)
  auto* s = new SnapshotGpu();
  s->tick = tick_; s->nb = nb_; s->cap = cap_b_ > nb_ ? cap_b_ : nb_; s->n_warm = n_warm;
  size_t n = nb_ + 1;
  s->pos.ensure(n); s->rot.ensure(n); s->lin.ensure(n); s->ang.ensure(n); s->last_lin.ensure(n);
  s->awake.ensure(s->cap + 1); s->ticks.ensure(s->cap + 1);
  s->wk.ensure(n_warm + 1); s->wa.ensure(n_warm + 1); s->wb.ensure(n_warm + 1);
  auto cp = [&](void* d, const void* src, size_t bytes) {
    if (bytes) RP_CUDA(cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, stream_));
  };
  cp(s->pos.p, pos.p, 16 * (size_t)nb_); cp(s->rot.p, rot.p, 16 * (size_t)nb_);
  cp(s->lin.p, lin.p, 16 * (size_t)nb_); cp(s->ang.p, ang.p, 16 * (size_t)nb_);
  cp(s->last_lin.p, last_lin.p, 16 * (size_t)nb_);
  cp(s->awake.p, awake.p, s->cap); cp(s->ticks.p, sleep_ticks.p, 2 * (size_t)s->cap);
  cp(s->wk.p, warm_key.p, 16 * (size_t)n_warm); cp(s->wa.p, warm_a.p, 16 * (size_t)n_warm);
  cp(s->wb.p, warm_b.p, 16 * (size_t)n_warm);
  upload_joints();
  s->nj = num_joints();
  s->jw_n.ensure(s->nj + 1); s->jw_tag.ensure(kJointRows * (size_t)s->nj + kJointRows); s->jw_lam.ensure(kJointRows * (size_t)s->nj + kJointRows);
  cp(s->jw_n.p, jw_n.p, 4 * (size_t)s->nj);
  cp(s->jw_tag.p, jw_tag.p, kJointRows * (size_t)s->nj);
  cp(s->jw_lam.p, jw_lam.p, 4 * kJointRows * (size_t)s->nj);
  RP_CUDA(cudaStreamSynchronize(stream_));
  s->players = players();
  return s;
}
// Every stored bit back (a World clone, not the FFI's pose injection): for rollback that must
// replay bit for bit. The body set must be the one the snapshot saw.
void WorldGpu::snapshot_restore_exact(const SnapshotGpu* s) {
  if (s->nb != nb_) throw std::invalid_argument("exact restore needs the body set of the snapshot");
  tick_ = s->tick;
  auto cp = [&](void* d, const void* src, size_t bytes) {
    if (bytes) RP_CUDA(cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, stream_));
  };
  cp(pos.p, s->pos.p, 16 * (size_t)nb_); cp(rot.p, s->rot.p, 16 * (size_t)nb_);
  cp(lin.p, s->lin.p, 16 * (size_t)nb_); cp(ang.p, s->ang.p, 16 * (size_t)nb_);
  cp(last_lin.p, s->last_lin.p, 16 * (size_t)nb_);
  uint32_t cap = cap_b_ > nb_ ? cap_b_ : nb_;
  uint32_t ncap = s->cap < cap ? s->cap : cap;
  cp(awake.p, s->awake.p, ncap); cp(sleep_ticks.p, s->ticks.p, 2 * (size_t)ncap);
  warm_key.ensure(s->n_warm + 1); warm_a.ensure(s->n_warm + 1); warm_b.ensure(s->n_warm + 1);
  cp(warm_key.p, s->wk.p, 16 * (size_t)s->n_warm); cp(warm_a.p, s->wa.p, 16 * (size_t)s->n_warm);
  cp(warm_b.p, s->wb.p, 16 * (size_t)s->n_warm);
  n_warm = s->n_warm;
  restore_joint_warm(s);
  RP_CUDA(cudaStreamSynchronize(stream_));
  set_players(s->players);
}
// The joint cache as the snapshot held it; joints added since have no entry.
void WorldGpu::restore_joint_warm(const SnapshotGpu* s) {
  upload_joints();
  uint32_t nj = num_joints(), n = s->nj < nj ? s->nj : nj;
  if (n) {
    RP_CUDA(cudaMemcpyAsync(jw_n.p, s->jw_n.p, 4 * (size_t)n, cudaMemcpyDeviceToDevice, stream_));
    RP_CUDA(cudaMemcpyAsync(jw_tag.p, s->jw_tag.p, kJointRows * (size_t)n, cudaMemcpyDeviceToDevice, stream_));
    RP_CUDA(cudaMemcpyAsync(jw_lam.p, s->jw_lam.p, 4 * kJointRows * (size_t)n, cudaMemcpyDeviceToDevice, stream_));
  }
  if (nj > n) RP_CUDA(cudaMemsetAsync(jw_n.p + n, 0xFF, 4 * (size_t)(nj - n), stream_));
}
void WorldGpu::snapshot_restore(const SnapshotGpu* s) {  // lib.rs:1754-1793 + restore_carried_state
  tick_ = s->tick;
  uint32_t n = s->nb < nb_ ? s->nb : nb_;
  const int T = 256;
  if (n) {
    k_restore_bodies<<<(n + T - 1) / T, T, 0, stream_>>>(n, s->pos.p, s->rot.p, s->lin.p, s->ang.p, s->last_lin.p,
                                                          alive_d.p, pos.p, rot.p, lin.p, ang.p, last_lin.p); RP_COUNT_LAUNCH(1);
  }
  uint32_t ncap = s->cap < (cap_b_ > nb_ ? cap_b_ : nb_) ? s->cap : (cap_b_ > nb_ ? cap_b_ : nb_);
  if (ncap) {
    RP_CUDA(cudaMemcpyAsync(awake.p, s->awake.p, ncap, cudaMemcpyDeviceToDevice, stream_));
    RP_CUDA(cudaMemcpyAsync(sleep_ticks.p, s->ticks.p, 2 * (size_t)ncap, cudaMemcpyDeviceToDevice, stream_));
  }
  warm_key.ensure(s->n_warm + 1); warm_a.ensure(s->n_warm + 1); warm_b.ensure(s->n_warm + 1);
  if (s->n_warm) {
    RP_CUDA(cudaMemcpyAsync(warm_key.p, s->wk.p, 16 * (size_t)s->n_warm, cudaMemcpyDeviceToDevice, stream_));
    RP_CUDA(cudaMemcpyAsync(warm_a.p, s->wa.p, 16 * (size_t)s->n_warm, cudaMemcpyDeviceToDevice, stream_));
    RP_CUDA(cudaMemcpyAsync(warm_b.p, s->wb.p, 16 * (size_t)s->n_warm, cudaMemcpyDeviceToDevice, stream_));
  }
  n_warm = s->n_warm;
  filter_warm(1, 0);
  restore_joint_warm(s);
  filter_joint_warm_alive();
  RP_CUDA(cudaStreamSynchronize(stream_));
  set_players(s->players);  // lib.rs:1775
}
void WorldGpu::snapshot_free(SnapshotGpu* s) { delete s; }

}  // namespace rp
