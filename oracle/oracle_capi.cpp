// oracle/oracle_capi.cpp -- TEST INFRASTRUCTURE (the oracle). The reference's C ABI
// (crates/riftphys-ffi/src/lib.rs) over the CPU restatement in oracle_world.cpp, exporting the
// same rphys_* symbols as the product library so one test suite drives both. Validation order,
// error codes, thread-local messages and deterministic out-param defaults follow lib.rs.
#include <climits>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "../include/rphys_ext.h"
#include "oracle_world.h"

using namespace orc;
using om::V3;
using om::Q4;

static thread_local std::string g_err;
static thread_local bool g_has_err = false;
static void clear_err() { g_has_err = false; g_err.clear(); }
static RPhysResult fail(RPhysResult code, const std::string& m) { g_err = m; g_has_err = true; return code; }

struct RPhysWorld {
  std::mutex mu;
  World w;
  uint32_t bodies_created = 0, colliders_created = 0, max_bodies, max_colliders;
  RPhysTuning tuning{64, 32, 128};
  RPhysWorld(uint32_t mb, uint32_t mc) : w(mb), max_bodies(mb), max_colliders(mc) {}
};
struct RPhysWorldSnapshot { Snapshot s; std::vector<World::Player> players; };  // lib.rs:1696-1702

static V3 v(const RPhysVec3& a) { return V3{a.x, a.y, a.z}; }
static Q4 q(const RPhysQuat& a) { return Q4{a.x, a.y, a.z, a.w}; }
static bool fin3(const RPhysVec3& a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
static bool fin_iso(const RPhysIsometry& p) {
  return fin3(p.pos) && std::isfinite(p.rot.x) && std::isfinite(p.rot.y) && std::isfinite(p.rot.z) && std::isfinite(p.rot.w);
}
static bool fin_vel(const RPhysVelocity& a) { return fin3(a.lin) && fin3(a.ang); }
static bool fin_mat(const RPhysMaterial& m) {
  return std::isfinite(m.mu_static) && std::isfinite(m.mu_dynamic) && std::isfinite(m.restitution);
}

// checked_live_body_id (lib.rs:373-409)
static RPhysResult live_id(RPhysWorld* W, uint32_t id, const char* ctx, uint32_t* out) {
  if (id == 0) return fail(RPHYS_ERR_INVALID_ID, std::string(ctx) + ": body_id == 0 (invalid)");
  if (id == RPHYS_TERRAIN_BODY_ID) return fail(RPHYS_ERR_INVALID_ID, std::string(ctx) + ": body_id is terrain sentinel (not a real body)");
  uint32_t raw = id - 1;
  if (raw >= W->bodies_created) return fail(RPHYS_ERR_INVALID_ID, std::string(ctx) + ": body_id out of range");
  if (!(raw < W->w.alive.size() && W->w.alive[raw])) return fail(RPHYS_ERR_INVALID_ID, std::string(ctx) + ": body_id not found (removed)");
  *out = raw;
  return RPHYS_OK;
}
static RPhysResult add_common(RPhysWorld* W, const char* ctx, const RPhysIsometry& pose, const RPhysVelocity& vel,
                              uint32_t shape, const float dims[3], float density, bool dynamic, uint32_t mat,
                              bool sleep_allowed, uint32_t* out_id) {
  if (W->bodies_created + 1ull > W->max_bodies) return fail(RPHYS_ERR_CAPACITY, std::string(ctx) + ": body capacity exceeded");
  if (W->colliders_created + 1ull > W->max_colliders) return fail(RPHYS_ERR_CAPACITY, std::string(ctx) + ": collider capacity exceeded");
  float im = 0; V3 inertia{0, 0, 0};
  if (dynamic) mass_from_density(shape, dims, density, &im, &inertia);
  Shape s{shape, dims[0], dims[1], dims[2], V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}};
  if (shape == SH_SPHERE) { s.b = 0; s.c = 0; }
  if (shape == SH_CAPSULE) { s.c = 0; }
  uint32_t id = W->w.add_body(Iso{v(pose.pos), q(pose.rot)}, v(vel.lin), v(vel.ang), im, inertia, dynamic);
  if (id != W->bodies_created) return fail(RPHYS_ERR_INTERNAL, std::string(ctx) + ": internal body id reuse/skip");
  W->bodies_created++;
  W->w.add_collider(id, s, mat);
  W->colliders_created++;
  if (!sleep_allowed) { W->w.sleep_allowed[id] = 0; W->w.wake(id); }
  *out_id = id + 1;
  return RPHYS_OK;
}

extern "C" {

uint32_t rphys_get_abi_version(void) { return RPHYS_ABI_VERSION; }
const char* rphys_get_build_id(void) { return "riftphys_ffi-oracle-0.1.0"; }
const char* rphys_last_error_message(void) { return g_has_err ? g_err.c_str() : nullptr; }

RPhysResult rphys_last_error_copy(char* dst, uint32_t cap, uint32_t* out_len) {
  uint32_t len = g_has_err ? (uint32_t)g_err.size() : 0;
  if (out_len) *out_len = len;
  if (cap == 0) return RPHYS_OK;
  if (!dst) return RPHYS_ERR_NULL;
  uint32_t n = len < cap - 1 ? len : cap - 1;
  if (n) std::memcpy(dst, g_err.data(), n);
  dst[n] = 0;
  return RPHYS_OK;
}

RPhysWorld* rphys_world_create(uint32_t max_bodies, uint32_t max_colliders) {
  clear_err();
  try { return new RPhysWorld(max_bodies, max_colliders); } catch (...) { fail(RPHYS_ERR_INTERNAL, "panic in rphys_world_create"); return nullptr; }
}
void rphys_world_destroy(RPhysWorld* w) { delete w; }

RPhysResult rphys_world_set_epoch(RPhysWorld* W, uint64_t e) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_world_set_epoch: world is null");
  std::lock_guard<std::mutex> g(W->mu); W->w.epoch = e; return RPHYS_OK;
}
RPhysResult rphys_world_set_rng_seed(RPhysWorld* W, uint64_t s) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_world_set_rng_seed: world is null");
  std::lock_guard<std::mutex> g(W->mu); W->w.rng = s | 1ull; return RPHYS_OK;
}

RPhysResult rphys_add_capsule_body(RPhysWorld* W, const RPhysCapsuleBodyDesc* d, uint32_t* out) {
  clear_err();
  const char* ctx = "rphys_add_capsule_body";
  if (out) *out = 0;
  if (!W || !d || !out) return fail(RPHYS_ERR_NULL, std::string(ctx) + ": null arg");
  if (!fin_iso(d->pose)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": pose contains NaN/Inf");
  if (!fin_vel(d->vel)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": vel contains NaN/Inf");
  if (!fin_mat(d->material)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": material contains NaN/Inf");
  if (!(std::isfinite(d->radius) && d->radius > 0)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": radius must be finite and > 0");
  if (!(std::isfinite(d->half_height) && d->half_height >= 0)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": half_height must be finite and >= 0");
  if (d->body_type > 1) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": invalid body_type");
  if (d->body_type == 1 && !(std::isfinite(d->mass) && d->mass > 0)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": dynamic body mass must be finite and > 0");
  std::lock_guard<std::mutex> g(W->mu);
  float dims[3] = {d->radius, d->half_height, 0};
  return add_common(W, ctx, d->pose, d->vel, SH_CAPSULE, dims, 1500.0f, d->body_type == 1, 0, true, out);
}
RPhysResult rphys_add_box_body(RPhysWorld* W, const RPhysBoxBodyDesc* d, uint32_t* out) {
  clear_err();
  const char* ctx = "rphys_add_box_body";
  if (out) *out = 0;
  if (!W || !d || !out) return fail(RPHYS_ERR_NULL, std::string(ctx) + ": null arg");
  if (!fin_iso(d->pose)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": pose contains NaN/Inf");
  if (!fin_vel(d->vel)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": vel contains NaN/Inf");
  if (!fin_mat(d->material)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": material contains NaN/Inf");
  if (!(std::isfinite(d->hx) && d->hx > 0)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": hx must be finite and > 0");
  if (!(std::isfinite(d->hy) && d->hy > 0)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": hy must be finite and > 0");
  if (!(std::isfinite(d->hz) && d->hz > 0)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": hz must be finite and > 0");
  if (d->body_type > 1) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": invalid body_type");
  if (d->body_type == 1 && !(std::isfinite(d->mass) && d->mass > 0)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": dynamic body mass must be finite and > 0");
  std::lock_guard<std::mutex> g(W->mu);
  float dims[3] = {d->hx, d->hy, d->hz};
  return add_common(W, ctx, d->pose, d->vel, SH_BOX, dims, 1500.0f, d->body_type == 1, 0, true, out);
}
RPhysResult rphys_add_sphere_body(RPhysWorld* W, const RPhysSphereBodyDesc* d, uint32_t* out) {
  clear_err();
  const char* ctx = "rphys_add_sphere_body";
  if (out) *out = 0;
  if (!W || !d || !out) return fail(RPHYS_ERR_NULL, std::string(ctx) + ": null arg");
  if (!fin_iso(d->pose)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": pose contains NaN/Inf");
  if (!fin_vel(d->vel)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": vel contains NaN/Inf");
  if (!fin_mat(d->material)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": material contains NaN/Inf");
  if (!(std::isfinite(d->radius) && d->radius > 0)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": radius must be finite and > 0");
  if (d->body_type > 1) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": invalid body_type");
  if (d->body_type == 1 && !(std::isfinite(d->mass) && d->mass > 0)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": dynamic body mass must be finite and > 0");
  std::lock_guard<std::mutex> g(W->mu);
  float dims[3] = {d->radius, 0, 0};
  return add_common(W, ctx, d->pose, d->vel, SH_SPHERE, dims, 1500.0f, d->body_type == 1, 0, true, out);
}
RPhysResult rphys_body_remove(RPhysWorld* W, uint32_t id) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_body_remove: world is null");
  std::lock_guard<std::mutex> g(W->mu);
  uint32_t b; RPhysResult r = live_id(W, id, "rphys_body_remove", &b);
  if (r) return r;
  if (!W->w.remove_body(b)) return fail(RPHYS_ERR_INTERNAL, "rphys_body_remove: internal remove failed");
  return RPHYS_OK;
}
RPhysResult rphys_body_get_pose(const RPhysWorld* Wc, uint32_t id, RPhysIsometry* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_body_get_pose: out_pose is null");
  *out = RPhysIsometry{{0, 0, 0}, {0, 0, 0, 1}};
  if (!Wc) return fail(RPHYS_ERR_NULL, "rphys_body_get_pose: world is null");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  uint32_t b; RPhysResult r = live_id(W, id, "rphys_body_get_pose", &b);
  if (r) return r;
  V3 p = W->w.pos[b]; Q4 o = W->w.rot[b];
  *out = RPhysIsometry{{p.x, p.y, p.z}, {o.x, o.y, o.z, o.w}};
  return RPHYS_OK;
}
RPhysResult rphys_body_set_pose(RPhysWorld* W, uint32_t id, const RPhysIsometry* p) {
  clear_err();
  if (!W || !p) return fail(RPHYS_ERR_NULL, "rphys_body_set_pose: null arg");
  if (!fin_iso(*p)) return fail(RPHYS_ERR_BAD_ARG, "rphys_body_set_pose: pose contains NaN/Inf");
  std::lock_guard<std::mutex> g(W->mu);
  uint32_t b; RPhysResult r = live_id(W, id, "rphys_body_set_pose", &b);
  if (r) return r;
  W->w.set_body_pose(b, Iso{v(p->pos), q(p->rot)});
  return RPHYS_OK;
}
RPhysResult rphys_body_get_velocity(const RPhysWorld* Wc, uint32_t id, RPhysVelocity* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_body_get_velocity: out_vel is null");
  *out = RPhysVelocity{{0, 0, 0}, {0, 0, 0}};
  if (!Wc) return fail(RPHYS_ERR_NULL, "rphys_body_get_velocity: world is null");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  uint32_t b; RPhysResult r = live_id(W, id, "rphys_body_get_velocity", &b);
  if (r) return r;
  V3 l = W->w.lin[b], a = W->w.ang[b];
  *out = RPhysVelocity{{l.x, l.y, l.z}, {a.x, a.y, a.z}};
  return RPHYS_OK;
}
RPhysResult rphys_body_set_velocity(RPhysWorld* W, uint32_t id, const RPhysVelocity* vel) {
  clear_err();
  if (!W || !vel) return fail(RPHYS_ERR_NULL, "rphys_body_set_velocity: null arg");
  if (!fin_vel(*vel)) return fail(RPHYS_ERR_BAD_ARG, "rphys_body_set_velocity: velocity contains NaN/Inf");
  std::lock_guard<std::mutex> g(W->mu);
  uint32_t b; RPhysResult r = live_id(W, id, "rphys_body_set_velocity", &b);
  if (r) return r;
  W->w.set_body_vel(b, v(vel->lin), v(vel->ang));
  return RPHYS_OK;
}
RPhysResult rphys_body_apply_impulse(RPhysWorld* W, uint32_t id, RPhysVec3 imp) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_body_apply_impulse: world is null");
  if (!fin3(imp)) return fail(RPHYS_ERR_BAD_ARG, "rphys_body_apply_impulse: impulse contains NaN/Inf");
  std::lock_guard<std::mutex> g(W->mu);
  uint32_t b; RPhysResult r = live_id(W, id, "rphys_body_apply_impulse", &b);
  if (r) return r;
  W->w.apply_impulse_world(b, v(imp));
  return RPHYS_OK;
}

RPhysResult rphys_world_step_ex(RPhysWorld* W, const RPhysStepParams* p) {
  clear_err();
  if (!W || !p) return fail(RPHYS_ERR_NULL, "rphys_world_step_ex: null arg");
  if (p->size_bytes < sizeof(RPhysStepParams)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_step_ex: size_bytes too small");
  if (!std::isfinite(p->dt)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_step_ex: dt is not finite");
  if (p->dt < 0) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_step_ex: dt is negative");
  if (p->substeps == 0) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_step_ex: substeps == 0");
  std::lock_guard<std::mutex> g(W->mu);
  float sub = p->dt / (float)p->substeps;
  if (!std::isfinite(sub)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_step_ex: sub_dt is not finite");
  for (uint32_t i = 0; i < p->substeps; ++i) W->w.step(sub);
  return RPHYS_OK;
}
RPhysResult rphys_world_step(RPhysWorld* W, float dt) {
  RPhysStepParams p{(uint32_t)sizeof(RPhysStepParams), 0, 1, 0, dt};
  return rphys_world_step_ex(W, &p);
}
RPhysResult rphys_world_tick_index(const RPhysWorld* Wc, uint64_t* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_world_tick_index: out_tick is null");
  *out = 0;
  if (!Wc) return fail(RPHYS_ERR_NULL, "rphys_world_tick_index: world is null");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  *out = W->w.tick;
  return RPHYS_OK;
}
RPhysResult rphys_world_num_bodies(const RPhysWorld* Wc, uint32_t* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_world_num_bodies: out_num is null");
  *out = 0;
  if (!Wc) return fail(RPHYS_ERR_NULL, "rphys_world_num_bodies: world is null");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  *out = W->w.num_bodies();
  return RPHYS_OK;
}
RPhysResult rphys_world_get_step_hash(const RPhysWorld* Wc, RPhysHash32* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_world_get_step_hash: out_hash is null");
  std::memset(out, 0, sizeof(*out));
  if (!Wc) return fail(RPHYS_ERR_NULL, "rphys_world_get_step_hash: world is null");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  W->w.step_hash(out->bytes);
  return RPHYS_OK;
}
// Batches are a property of the CUDA library; the restatement steps each world as its own World
// (the tests build one oracle World per batch world), so these entry points only exist for the
// shared bindings.
RPhysResult rphys_ext_batch_add_world(RPhysWorld*, const RPhysBodyDescEx*, uint32_t, uint32_t* w, uint32_t* f) {
  if (w) *w = 0;
  if (f) *f = 0;
  return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_batch_add_world: the CPU restatement steps one world per RPhysWorld");
}
RPhysResult rphys_ext_batch_num_worlds(const RPhysWorld* W, uint32_t* out) {
  if (!W || !out) return fail(RPHYS_ERR_NULL, "rphys_ext_batch_num_worlds: null arg");
  *out = 1;
  return RPHYS_OK;
}
RPhysResult rphys_ext_batch_world_range(const RPhysWorld* W, uint32_t world, uint32_t* first, uint32_t* count) {
  if (!W || !first || !count) return fail(RPHYS_ERR_NULL, "rphys_ext_batch_world_range: null arg");
  if (world != 0) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_batch_world_range: no such world");
  *first = 1;
  *count = W->w.num_bodies();
  return RPHYS_OK;
}
RPhysResult rphys_ext_batch_get_hashes(const RPhysWorld* W, uint32_t first, uint32_t count, RPhysHash32* out) {
  if (!W || (!out && count)) return fail(RPHYS_ERR_NULL, "rphys_ext_batch_get_hashes: null arg");
  if ((uint64_t)first + count > 1) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_batch_get_hashes: world range out of bounds");
  for (uint32_t k = 0; k < count; ++k) rphys_world_get_step_hash(W, &out[k]);
  return RPHYS_OK;
}
// The CPU restatement allocates as it likes; this entry point only mirrors the CUDA library's
// symbol so both load through the same bindings, and returns the same digest.
RPhysResult rphys_ext_world_step_hash_noalloc(const RPhysWorld* Wc, RPhysHash32* out) {
  return rphys_world_get_step_hash(Wc, out);
}
RPhysResult rphys_world_step_and_hash(RPhysWorld* W, float dt, RPhysHash32* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_world_step_and_hash: out_hash is null");
  std::memset(out, 0, sizeof(*out));
  RPhysResult r = rphys_world_step(W, dt);
  if (r) return r;
  return rphys_world_get_step_hash(W, out);
}

static RPhysResult set_hf(RPhysWorld* W, uint32_t nx, uint32_t nz, float cx, float cz, float ox, float oz,
                          std::vector<float> h, uint32_t mat) {
  // HeightField::from_heights (terrain.rs:24-50)
  HeightField hf;
  hf.nx = nx; hf.nz = nz;
  hf.sx = (std::isfinite(cx) && cx > 0) ? om::q6(cx) : 1.0f;
  hf.sz = (std::isfinite(cz) && cz > 0) ? om::q6(cz) : 1.0f;
  hf.ox = ox; hf.oz = oz;
  float mn = INFINITY, mx = -INFINITY;
  for (auto& x : h) { float val = std::isfinite(x) ? x : 0.0f; x = om::q6(val); mn = om::rmin(mn, x); mx = om::rmax(mx, x); }
  hf.min_y = om::q6(mn); hf.max_y = om::q6(mx);
  hf.h = std::move(h);
  hf.mat = mat;
  W->w.hf = std::move(hf);
  W->w.has_hf = true;
  return RPHYS_OK;
}
RPhysResult rphys_world_set_heightfield_i16(RPhysWorld* W, const RPhysHeightfieldDesc* d, float ox, float oz, float yoff) {
  clear_err();
  if (!W || !d) return fail(RPHYS_ERR_NULL, "rphys_world_set_heightfield_i16: null arg");
  if (d->size_bytes < sizeof(RPhysHeightfieldDesc)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_set_heightfield_i16: size_bytes too small");
  if (d->width == 0 || d->height == 0) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_set_heightfield_i16: width/height == 0");
  if (d->row_stride != 0 && d->row_stride < d->width) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_set_heightfield_i16: row_stride must be >= width");
  if (!d->heights) return fail(RPHYS_ERR_NULL, "rphys_world_set_heightfield_i16: heights is null");
  if (!(std::isfinite(d->cell_size_x) && std::isfinite(d->cell_size_z) && d->cell_size_x > 0 && d->cell_size_z > 0))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_world_set_heightfield_i16: bad cell sizes");
  uint32_t stride = d->row_stride == 0 ? d->width : d->row_stride;
  std::vector<float> h;
  h.reserve((size_t)d->width * d->height);
  for (uint32_t r = 0; r < d->height; ++r)
    for (uint32_t c = 0; c < d->width; ++c)
      h.push_back(((float)d->heights[(size_t)r * stride + c] * d->height_scale + d->height_offset) + yoff);
  std::lock_guard<std::mutex> g(W->mu);
  return set_hf(W, d->width, d->height, d->cell_size_x, d->cell_size_z, ox, oz, std::move(h), 4);
}
RPhysResult rphys_world_set_heightfield_raw32_square(RPhysWorld* W, const uint8_t* bytes, uint32_t n, float wx, float wz,
                                                     float ox, float oz, float yoff) {
  clear_err();
  if (!W || !bytes) return fail(RPHYS_ERR_NULL, "rphys_world_set_heightfield_raw32_square: null arg");
  if (n < 4) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_set_heightfield_raw32_square: bytes_len too small to form a grid");
  size_t cnt = n / 4;
  size_t dim = (size_t)std::sqrt((double)cnt);
  if (dim * dim != cnt) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_set_heightfield_raw32_square: byte length is not a square number of f32s");
  float cx = wx / om::rmax((float)dim - 1.0f, 1.0f), cz = wz / om::rmax((float)dim - 1.0f, 1.0f);
  std::vector<float> h(cnt);
  for (size_t i = 0; i < cnt; ++i) { float x; std::memcpy(&x, bytes + 4 * i, 4); h[i] = x + yoff; }
  std::lock_guard<std::mutex> g(W->mu);
  return set_hf(W, (uint32_t)dim, (uint32_t)dim, cx, cz, ox, oz, std::move(h), 4);
}
RPhysResult rphys_world_clear_heightfield(RPhysWorld* W) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_world_clear_heightfield: world is null");
  std::lock_guard<std::mutex> g(W->mu);
  W->w.has_hf = false;
  W->w.hf = HeightField{};
  return RPHYS_OK;
}

// pack_snapshot (riftphys-riftnet/src/wire.rs:36-53) over every live body in id order; the entity
// scale from the body's collider as wire.rs:22-23 defines it.
RPhysResult rphys_ext_pack_snapshot(RPhysWorld* W, uint64_t tick, uint64_t epoch, uint8_t* out, uint64_t out_cap,
                                    uint64_t* out_bytes, uint32_t* out_chunks) {
  clear_err();
  if (out_bytes) *out_bytes = 0;
  if (out_chunks) *out_chunks = 0;
  if (!W || !out_bytes || !out_chunks) return fail(RPHYS_ERR_NULL, "rphys_ext_pack_snapshot: null arg");
  std::lock_guard<std::mutex> g(W->mu);
  const uint32_t per = 1200u / 48u;
  std::vector<uint32_t> live;
  for (uint32_t i = 0; i < W->w.num_bodies(); ++i)
    if (W->w.alive[i]) live.push_back(i);
  const uint32_t n = (uint32_t)live.size(), chunks = (n + per - 1) / per;
  const uint64_t bytes = (uint64_t)chunks * 32u + (uint64_t)n * 48u;
  *out_bytes = bytes;
  *out_chunks = chunks;
  if (!out) return RPHYS_OK;
  if (out_cap < bytes) return fail(RPHYS_ERR_CAPACITY, "rphys_ext_pack_snapshot: buffer smaller than the snapshot");
  uint8_t* p = out;
  for (uint32_t c = 0; c < chunks; ++c) {
    const uint32_t k = std::min(per, n - c * per);
    uint8_t hdr[32] = {};
    const uint32_t magic = 0x30535052u, plen = k * 48u;
    const uint16_t ver = 2, total = (uint16_t)chunks, index = (uint16_t)c;
    std::memcpy(hdr + 0, &magic, 4); std::memcpy(hdr + 4, &ver, 2); hdr[6] = 1; hdr[7] = 0;
    std::memcpy(hdr + 8, &tick, 8); std::memcpy(hdr + 16, &epoch, 8);
    std::memcpy(hdr + 24, &total, 2); std::memcpy(hdr + 26, &index, 2); std::memcpy(hdr + 28, &plen, 4);
    std::memcpy(p, hdr, 32);
    p += 32;
    for (uint32_t e = c * per; e < c * per + k; ++e) {
      const uint32_t b = live[e];
      const orc::Shape& sh = W->w.colliders[b].shape;
      float ent[12];
      uint32_t id = b + 1, kind;
      float sx, sy, sz;
      if (sh.kind == SH_SPHERE) { sx = sy = sz = sh.a; kind = 1; }
      else if (sh.kind == SH_BOX) { sx = sh.a; sy = sh.b; sz = sh.c; kind = 2; }
      else { sx = sh.a; sy = (sh.b + sh.a) * 0.5f; sz = sh.a; kind = 3; }
      std::memcpy(ent + 0, &id, 4);
      ent[1] = W->w.pos[b].x; ent[2] = W->w.pos[b].y; ent[3] = W->w.pos[b].z;
      ent[4] = W->w.rot[b].x; ent[5] = W->w.rot[b].y; ent[6] = W->w.rot[b].z; ent[7] = W->w.rot[b].w;
      ent[8] = sx; ent[9] = sy; ent[10] = sz;
      std::memcpy(ent + 11, &kind, 4);
      std::memcpy(p, ent, 48);
      p += 48;
    }
  }
  return RPHYS_OK;
}
// rphys_world_raycast (riftphys-ffi/src/lib.rs:1271-1346, 470-479)
static void write_raycast_miss(RPhysRayHit* h) {
  h->hit = RPHYS_FALSE;
  h->body_id = RPHYS_INVALID_BODY_ID;
  h->fraction = 1.0f;
  h->point = RPhysVec3{0.0f, 0.0f, 0.0f};
  h->normal = RPhysVec3{0.0f, 1.0f, 0.0f};
}
static RPhysResult raycast_one(RPhysWorld* W, const RPhysRayQuery& q, const char* ctx, RPhysRayHit* out, bool exact = false) {
  write_raycast_miss(out);
  auto fin3 = [](RPhysVec3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); };
  if (!fin3(q.origin)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": origin contains NaN/Inf");
  if (!fin3(q.dir)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": dir contains NaN/Inf");
  if (!std::isfinite(q.max_distance)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": max_distance is not finite");
  uint32_t ignore = 0xFFFFFFFFu;
  if (q.ignore_body != 0) {
    const std::string ictx = std::string(ctx) + ".ignore_body";
    RPhysResult r = live_id(W, q.ignore_body, ictx.c_str(), &ignore);
    if (r) return r;
  }
  if (q.max_distance <= 0.0f) return RPHYS_OK;
  V3 d = v(q.dir);
  const float len2 = om::dot(d, d);
  if (!std::isfinite(len2)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": dir length overflow/invalid");
  if (len2 <= 1.0e-20f) return RPHYS_OK;
  d = om::divs(d, std::sqrt(len2));
  uint32_t body;
  float toi;
  V3 p, n;
  const bool hit = exact ? W->w.raycast_exact(v(q.origin), d, q.max_distance, ignore, &body, &toi, &p, &n)
                         : W->w.raycast(v(q.origin), d, q.max_distance, ignore, &body, &toi, &p, &n);
  if (!hit) return RPHYS_OK;
  out->hit = RPHYS_TRUE;
  out->body_id = body == 0xFFFFFFFFu ? RPHYS_TERRAIN_BODY_ID : body + 1;
  out->fraction = om::clampf(toi, 0.0f, 1.0f);
  out->point = RPhysVec3{p.x, p.y, p.z};
  out->normal = RPhysVec3{n.x, n.y, n.z};
  return RPHYS_OK;
}
RPhysResult rphys_world_raycast(const RPhysWorld* Wc, const RPhysRayQuery* q, RPhysRayHit* out) {
  clear_err();
  if (out) write_raycast_miss(out);
  if (!Wc || !q || !out) return fail(RPHYS_ERR_NULL, "rphys_world_raycast: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  return raycast_one(W, *q, "rphys_world_raycast", out);
}
RPhysResult rphys_ext_raycast_batch(const RPhysWorld* Wc, const RPhysRayQuery* q, uint32_t n, RPhysRayHit* out) {
  clear_err();
  if (!Wc || ((!q || !out) && n)) return fail(RPHYS_ERR_NULL, "rphys_ext_raycast_batch: null arg");
  for (uint32_t i = 0; i < n; ++i) write_raycast_miss(out + i);
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  for (uint32_t i = 0; i < n; ++i) {
    RPhysResult r = raycast_one(W, q[i], "rphys_ext_raycast_batch", out + i);
    if (r) {
      for (uint32_t k = 0; k < n; ++k) write_raycast_miss(out + k);
      return r;
    }
  }
  return RPHYS_OK;
}
// rphys_world_capsule_sweep (riftphys-ffi/src/lib.rs:1349-1411, 482-492)
// World::raycast_exact (queries.rs:18-48) for n rays, checked and normalised as rphys_world_raycast
RPhysResult rphys_ext_raycast_exact_batch(const RPhysWorld* Wc, const RPhysRayQuery* q, uint32_t n, RPhysRayHit* out) {
  clear_err();
  if (!Wc || ((!q || !out) && n)) return fail(RPHYS_ERR_NULL, "rphys_ext_raycast_exact_batch: null arg");
  for (uint32_t i = 0; i < n; ++i) write_raycast_miss(out + i);
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  for (uint32_t i = 0; i < n; ++i) {
    RPhysResult r = raycast_one(W, q[i], "rphys_ext_raycast_exact_batch", out + i, true);
    if (r) {
      for (uint32_t k = 0; k < n; ++k) write_raycast_miss(out + k);
      return r;
    }
  }
  return RPHYS_OK;
}
RPhysResult rphys_world_capsule_sweep(const RPhysWorld* Wc, const RPhysCapsuleSweepQuery* q, RPhysCapsuleSweepHit* out) {
  clear_err();
  if (out) {
    out->hit = RPHYS_FALSE; out->body_id = RPHYS_INVALID_BODY_ID; out->fraction = 1.0f; out->started_overlapping = RPHYS_FALSE;
    out->point = RPhysVec3{0.0f, 0.0f, 0.0f}; out->normal = RPhysVec3{0.0f, 1.0f, 0.0f};
  }
  if (!Wc || !q || !out) return fail(RPHYS_ERR_NULL, "rphys_world_capsule_sweep: null arg");
  auto fin3 = [](RPhysVec3 a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); };
  if (!fin3(q->from)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_capsule_sweep: from contains NaN/Inf");
  if (!fin3(q->to)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_capsule_sweep: to contains NaN/Inf");
  if (!(std::isfinite(q->radius) && q->radius > 0.0f))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_world_capsule_sweep: radius must be finite and > 0");
  if (!(std::isfinite(q->half_height) && q->half_height >= 0.0f))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_world_capsule_sweep: half_height must be finite and >= 0");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  uint32_t ignore = 0xFFFFFFFFu;
  if (q->ignore_body != 0) {
    RPhysResult r = live_id(W, q->ignore_body, "rphys_world_capsule_sweep.ignore_body", &ignore);
    if (r) return r;
  }
  uint32_t body;
  float toi;
  bool overlap;
  V3 p, n;
  if (!W->w.sweep_capsule(v(q->from), v(q->to), q->radius, q->half_height, ignore, &body, &toi, &overlap, &p, &n))
    return RPHYS_OK;
  out->hit = RPHYS_TRUE;
  out->body_id = body == 0xFFFFFFFFu ? RPHYS_TERRAIN_BODY_ID : body + 1;
  out->fraction = om::clampf(toi, 0.0f, 1.0f);
  out->started_overlapping = overlap ? RPHYS_TRUE : RPHYS_FALSE;
  out->point = RPhysVec3{p.x, p.y, p.z};
  out->normal = RPhysVec3{n.x, n.y, n.z};
  return RPHYS_OK;
}

// rphys_add_player (lib.rs:1580-1627): the desc is checked before the lock, then one body and one
// collider of capacity; the controller gets the desc's size and speed after World::add_player.
RPhysResult rphys_add_player(RPhysWorld* W, const RPhysPlayerDesc* d, uint32_t* out) {
  clear_err();
  if (out) *out = 0xFFFFFFFFu;
  if (!W || !d || !out) return fail(RPHYS_ERR_NULL, "rphys_add_player: null arg");
  if (!fin_iso(d->start_pose)) return fail(RPHYS_ERR_BAD_ARG, "rphys_add_player: pose contains NaN/Inf");
  if (!(std::isfinite(d->radius) && d->radius > 0.0f)) return fail(RPHYS_ERR_BAD_ARG, "rphys_add_player: radius must be > 0");
  if (!(std::isfinite(d->height) && d->height > 0.0f)) return fail(RPHYS_ERR_BAD_ARG, "rphys_add_player: height must be > 0");
  std::lock_guard<std::mutex> g(W->mu);
  if (W->bodies_created + 1ull > W->max_bodies) return fail(RPHYS_ERR_CAPACITY, "rphys_add_player: body capacity exceeded");
  if (W->colliders_created + 1ull > W->max_colliders) return fail(RPHYS_ERR_CAPACITY, "rphys_add_player: collider capacity exceeded");
  const uint32_t idx = W->w.add_player(Iso{v(d->start_pose.pos), q(d->start_pose.rot)});
  W->bodies_created++;
  W->colliders_created++;
  World::Player& p = W->w.players[idx];
  p.radius = d->radius; p.height = d->height; p.speed = d->speed;
  *out = idx;
  return RPHYS_OK;
}
// rphys_player_get_pose (lib.rs:1629-1666): identity and false written first
RPhysResult rphys_player_get_pose(const RPhysWorld* Wc, uint32_t idx, RPhysIsometry* out, RPhysBool* grounded) {
  clear_err();
  if (out) *out = RPhysIsometry{RPhysVec3{0, 0, 0}, RPhysQuat{0, 0, 0, 1}};
  if (grounded) *grounded = RPHYS_FALSE;
  if (!Wc || !out) return RPHYS_ERR_NULL;
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  if (idx >= W->w.players.size()) return fail(RPHYS_ERR_BAD_ARG, "rphys_player_get_pose: player_idx out of bounds");
  const World::Player& p = W->w.players[idx];
  const V3 pp = W->w.pos[p.body];
  const Q4 qq = W->w.rot[p.body];
  *out = RPhysIsometry{RPhysVec3{pp.x, pp.y, pp.z}, RPhysQuat{qq.x, qq.y, qq.z, qq.w}};
  if (grounded) *grounded = p.grounded ? RPHYS_TRUE : RPHYS_FALSE;
  return RPHYS_OK;
}
// rphys_player_set_input (lib.rs:1668-1693)
RPhysResult rphys_player_set_input(RPhysWorld* W, uint32_t idx, RPhysVec3 dir) {
  clear_err();
  if (!W) return RPHYS_ERR_NULL;
  if (!fin3(dir)) return fail(RPHYS_ERR_BAD_ARG, "rphys_player_set_input: move_dir NaN/Inf");
  std::lock_guard<std::mutex> g(W->mu);
  if (idx >= W->w.players.size()) return fail(RPHYS_ERR_BAD_ARG, "rphys_player_set_input: player_idx out of bounds");
  W->w.players[idx].input = v(dir);
  return RPHYS_OK;
}
RPhysResult rphys_world_get_contacts(const RPhysWorld* Wc, RPhysContactEvent* out, uint32_t cap, uint32_t* out_count) {
  clear_err();
  if (!Wc || !out_count) return fail(RPHYS_ERR_NULL, "rphys_world_get_contacts: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  auto& cs = W->w.last_frame_contacts;
  *out_count = (uint32_t)cs.size();
  if (!out) return RPHYS_OK;
  uint32_t n = (uint32_t)cs.size() < cap ? (uint32_t)cs.size() : cap;
  for (uint32_t i = 0; i < n; ++i) {
    const Contact& c = cs[i];
    RPhysContactEvent e;
    e.body_id_a = W->w.colliders[c.a_collider].body + 1;
    e.body_id_b = c.b_collider == kTerrain ? RPHYS_TERRAIN_BODY_ID : W->w.colliders[c.b_collider].body + 1;
    e.position = RPhysVec3{c.point.x, c.point.y, c.point.z};
    e.normal = RPhysVec3{c.normal.x, c.normal.y, c.normal.z};
    e.impulse = c.impulse;
    out[i] = e;
  }
  return RPHYS_OK;
}

RPhysWorldSnapshot* rphys_world_snapshot_create(const RPhysWorld* Wc) {
  clear_err();
  if (!Wc) { fail(RPHYS_ERR_NULL, "rphys_world_snapshot_create: world is null"); return nullptr; }
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  auto* s = new RPhysWorldSnapshot();
  World& w = W->w;
  s->s.tick = w.tick;
  for (uint32_t i = 0; i < w.num_bodies(); ++i) {
    if (w.alive[i]) { s->s.poses.push_back(Iso{w.pos[i], w.rot[i]}); s->s.lin.push_back(w.lin[i]); s->s.ang.push_back(w.ang[i]); }
    else { s->s.poses.push_back(Iso{V3{0, 0, 0}, Q4{0, 0, 0, 1}}); s->s.lin.push_back(V3{0, 0, 0}); s->s.ang.push_back(V3{0, 0, 0}); }
  }
  s->s.carried = w.carried_state();
  s->players = w.players;
  return s;
}
RPhysResult rphys_world_snapshot_restore(RPhysWorld* W, const RPhysWorldSnapshot* s) {
  clear_err();
  if (!W || !s) return fail(RPHYS_ERR_NULL, "rphys_world_snapshot_restore: null arg");
  std::lock_guard<std::mutex> g(W->mu);
  World& w = W->w;
  w.tick = s->s.tick;
  w.players = s->players;  // lib.rs:1775
  for (uint32_t i = 0; i < s->s.poses.size(); ++i) {
    if (i < w.alive.size() && w.alive[i] && i < w.num_bodies()) {
      w.set_body_pose(i, s->s.poses[i]);
      w.set_body_vel(i, s->s.lin[i], s->s.ang[i]);
    }
  }
  w.restore_carried_state(s->s.carried);
  return RPHYS_OK;
}
// World-clone restore: the stored bits themselves, then the carried state.
RPhysResult rphys_ext_snapshot_restore_exact(RPhysWorld* W, const RPhysWorldSnapshot* s) {
  clear_err();
  if (!W || !s) return fail(RPHYS_ERR_NULL, "rphys_ext_snapshot_restore_exact: null arg");
  std::lock_guard<std::mutex> g(W->mu);
  World& w = W->w;
  if (s->s.poses.size() != w.num_bodies())
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_snapshot_restore_exact: bodies were added since the snapshot");
  w.tick = s->s.tick;
  for (uint32_t i = 0; i < w.num_bodies(); ++i) {
    w.pos[i] = s->s.poses[i].pos;
    w.rot[i] = s->s.poses[i].rot;
    w.lin[i] = s->s.lin[i];
    w.ang[i] = s->s.ang[i];
  }
  w.players = s->players;
  w.update_colliders_aabb();  // a world clone holds the AABBs of the stored poses
  w.restore_carried_state(s->s.carried);
  return RPHYS_OK;
}
// The state blob of rphys_ext_state_export (layout in rphys_ext.h): the same fields the device
// library writes, from the World's own containers.
static constexpr uint32_t kStateMagic = 0x31535052u;  // "RPS1"
static uint64_t state_size(const World& w) {
  uint64_t nb = w.num_bodies(), cap = w.awake.size() > nb ? w.awake.size() : nb, nw = 0;
  for (const auto& kv : w.warm) nw += kv.second.size();
  return 48 + 65 * nb + 3 * cap + 44 * nw + 164 * (uint64_t)w.joints.size();
}
RPhysResult rphys_ext_state_export(const RPhysWorld* Wc, uint8_t* out, uint64_t out_cap, uint64_t* out_bytes) {
  clear_err();
  if (!Wc || !out_bytes) return fail(RPHYS_ERR_NULL, "rphys_ext_state_export: null arg");
  *out_bytes = 0;
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  const World& w = W->w;
  if (!w.players.empty()) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_state_export: a world with players has no state blob");
  const uint64_t n = state_size(w);
  *out_bytes = n;
  if (!out) return RPHYS_OK;
  if (out_cap < n) return fail(RPHYS_ERR_CAPACITY, "rphys_ext_state_export: buffer smaller than the state");
  const uint32_t nb = w.num_bodies(), cap = (uint32_t)(w.awake.size() > nb ? w.awake.size() : nb);
  uint32_t nw = 0;
  for (const auto& kv : w.warm) nw += (uint32_t)kv.second.size();
  uint8_t* p = out;
  auto put = [&](const void* v, size_t b) { std::memcpy(p, v, b); p += b; };
  const uint32_t hdr[2] = {kStateMagic, 1u};
  put(hdr, 8); put(&w.tick, 8); put(&w.epoch, 8); put(&w.rng, 8);
  const uint32_t cnt[4] = {nb, cap, nw, (uint32_t)w.joints.size()};
  put(cnt, 16);
  for (uint32_t i = 0; i < nb; ++i) {
    const V3 ll = i < w.last_lin_vel.size() ? w.last_lin_vel[i] : V3{0, 0, 0};
    const float v[16] = {w.pos[i].x, w.pos[i].y, w.pos[i].z, w.rot[i].x, w.rot[i].y, w.rot[i].z, w.rot[i].w, w.lin[i].x,
                         w.lin[i].y, w.lin[i].z, w.ang[i].x, w.ang[i].y, w.ang[i].z, ll.x, ll.y, ll.z};
    put(v, 64);
  }
  for (uint32_t i = 0; i < nb; ++i) put(&w.alive[i], 1);
  for (uint32_t i = 0; i < cap; ++i) { uint8_t a = i < w.awake.size() ? w.awake[i] : 1; put(&a, 1); }
  for (uint32_t i = 0; i < cap; ++i) { uint16_t t = i < w.sleep_ticks.size() ? w.sleep_ticks[i] : 0; put(&t, 2); }
  for (const auto& kv : w.warm) {
    const uint32_t key[4] = {std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first), std::get<3>(kv.first)};
    for (const WarmContact& c : kv.second) {
      put(key, 16);
      const float v[7] = {c.la.x, c.la.y, c.la.z, c.jn, c.jt.x, c.jt.y, c.jt.z};
      put(v, 28);
    }
  }
  for (uint32_t j = 0; j < (uint32_t)w.joints.size(); ++j) {
    uint8_t rec[164];
    std::memset(rec, 0, sizeof(rec));
    uint32_t c = 0xFFFFFFFFu;
    auto it = w.warm_joints.find(j);
    if (it != w.warm_joints.end()) {
      if (it->second.size() > 32) return fail(RPHYS_ERR_INTERNAL, "rphys_ext_state_export: joint with more than 32 cached rows");
      c = (uint32_t)it->second.size();
      for (uint32_t k = 0; k < c; ++k) {
        rec[4 + k] = it->second[k].first;
        std::memcpy(rec + 36 + 4 * k, &it->second[k].second, 4);
      }
    }
    std::memcpy(rec, &c, 4);
    put(rec, 164);
  }
  return RPHYS_OK;
}
RPhysResult rphys_ext_state_import(RPhysWorld* W, const uint8_t* in, uint64_t bytes) {
  clear_err();
  if (!W || !in) return fail(RPHYS_ERR_NULL, "rphys_ext_state_import: null arg");
  std::lock_guard<std::mutex> g(W->mu);
  World& w = W->w;
  if (bytes < 48) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_state_import: state blob shorter than its header");
  uint32_t hdr[2], cnt[4];
  uint64_t tick, epoch, rng;
  std::memcpy(hdr, in, 8);
  if (hdr[0] != kStateMagic || hdr[1] != 1u) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_state_import: not a version 1 state blob");
  std::memcpy(&tick, in + 8, 8); std::memcpy(&epoch, in + 16, 8); std::memcpy(&rng, in + 24, 8);
  std::memcpy(cnt, in + 32, 16);
  const uint32_t nb = w.num_bodies(), cap = (uint32_t)(w.awake.size() > nb ? w.awake.size() : nb);
  const uint32_t nj = (uint32_t)w.joints.size(), nw = cnt[2];
  if (cnt[0] != nb || cnt[1] != cap || cnt[3] != nj)
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_state_import: state blob of another world");
  if (bytes != 48 + 65ull * nb + 3ull * cap + 44ull * nw + 164ull * nj)
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_state_import: state blob size does not match its counts");
  if (!w.players.empty()) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_state_import: a world with players takes no state blob");
  const uint8_t* p = in + 48 + 64ull * nb;
  for (uint32_t i = 0; i < nb; ++i)
    if (p[i] != w.alive[i]) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_state_import: state blob's live bodies differ from this world's");
  p = in + 48;
  if (w.last_lin_vel.size() < nb) w.last_lin_vel.resize(nb, V3{0, 0, 0});
  for (uint32_t i = 0; i < nb; ++i, p += 64) {
    float v[16];
    std::memcpy(v, p, 64);
    w.pos[i] = V3{v[0], v[1], v[2]}; w.rot[i] = Q4{v[3], v[4], v[5], v[6]};
    w.lin[i] = V3{v[7], v[8], v[9]}; w.ang[i] = V3{v[10], v[11], v[12]};
    w.last_lin_vel[i] = V3{v[13], v[14], v[15]};
  }
  p += nb;
  w.awake.resize(cap); w.sleep_ticks.resize(cap);
  for (uint32_t i = 0; i < cap; ++i) w.awake[i] = p[i];
  p += cap;
  for (uint32_t i = 0; i < cap; ++i) std::memcpy(&w.sleep_ticks[i], p + 2 * i, 2);
  p += 2ull * cap;
  w.warm.clear();
  for (uint32_t e = 0; e < nw; ++e, p += 44) {
    uint32_t key[4];
    float v[7];
    std::memcpy(key, p, 16);
    std::memcpy(v, p + 16, 28);
    w.warm[WarmKey{key[0], key[1], key[2], key[3]}].push_back(WarmContact{V3{v[0], v[1], v[2]}, v[3], V3{v[4], v[5], v[6]}});
  }
  w.warm_joints.clear();
  for (uint32_t j = 0; j < nj; ++j, p += 164) {
    uint32_t c;
    std::memcpy(&c, p, 4);
    if (c == 0xFFFFFFFFu) continue;
    WarmJointRows rows;
    for (uint32_t k = 0; k < c && k < 32; ++k) {
      float l;
      std::memcpy(&l, p + 36 + 4 * k, 4);
      rows.emplace_back(p[4 + k], l);
    }
    w.warm_joints[j] = rows;
  }
  w.tick = tick; w.epoch = epoch; w.rng = rng;
  w.update_colliders_aabb();
  return RPHYS_OK;
}
void rphys_world_snapshot_free(RPhysWorldSnapshot* s) { delete s; }

// ---------------------------------------------------------------- extensions
RPhysResult rphys_ext_add_bodies(RPhysWorld* W, const RPhysBodyDescEx* d, uint32_t n, uint32_t* out_first) {
  clear_err();
  if (out_first) *out_first = 0;
  if (!W || (!d && n) || !out_first) return fail(RPHYS_ERR_NULL, "rphys_ext_add_bodies: null arg");
  std::lock_guard<std::mutex> g(W->mu);
  if ((uint64_t)W->bodies_created + n > W->max_bodies) return fail(RPHYS_ERR_CAPACITY, "rphys_ext_add_bodies: body capacity exceeded");
  if ((uint64_t)W->colliders_created + n > W->max_colliders) return fail(RPHYS_ERR_CAPACITY, "rphys_ext_add_bodies: collider capacity exceeded");
  for (uint32_t i = 0; i < n; ++i) {
    const RPhysBodyDescEx& e = d[i];
    if (!fin_iso(e.pose) || !fin_vel(e.vel)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_bodies: pose/vel contains NaN/Inf");
    if (e.shape > 2 || e.body_type > 1 || !material_known(e.material_id)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_bodies: bad shape/body_type/material");
    int nd = e.shape == 0 ? 1 : (e.shape == 1 ? 3 : 1);
    for (int k = 0; k < nd; ++k) if (!(std::isfinite(e.dims[k]) && e.dims[k] > 0)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_bodies: dims must be finite and > 0");
    if (e.shape == 2 && !(std::isfinite(e.dims[1]) && e.dims[1] >= 0)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_bodies: half_height must be finite and >= 0");
    if (e.body_type == 1 && !(std::isfinite(e.density) && e.density > 0)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_bodies: density must be finite and > 0");
  }
  for (uint32_t i = 0; i < n; ++i) {
    const RPhysBodyDescEx& e = d[i];
    uint32_t id;
    RPhysResult r = add_common(W, "rphys_ext_add_bodies", e.pose, e.vel, e.shape, e.dims, e.density, e.body_type == 1,
                               e.material_id, e.sleep_allowed != 0, &id);
    if (r) return r;
    if (i == 0) *out_first = id;
  }
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_pair_props(RPhysWorld* W, uint32_t a, uint32_t b, const RPhysPairProps* p) {
  clear_err();
  if (!W || !p) return fail(RPHYS_ERR_NULL, "rphys_ext_set_pair_props: null arg");
  if (!material_known(a) || !material_known(b)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_pair_props: unknown material");
  if (!(std::isfinite(p->mu_s) && std::isfinite(p->mu_k) && std::isfinite(p->restitution) && std::isfinite(p->stribeck_v)))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_pair_props: non-finite property");
  std::lock_guard<std::mutex> g(W->mu);
  W->w.set_pair_props(a, b, PairProps{p->mu_s, p->mu_k, p->restitution, p->stribeck_v, 0.0f});
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_solver_iterations(RPhysWorld* W, uint32_t v_it, uint32_t p_it) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_solver_iterations: world is null");
  std::lock_guard<std::mutex> g(W->mu);
  W->w.iters_v = v_it < 1 ? 1 : v_it;
  W->w.iters_p = p_it < 1 ? 1 : p_it;
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_gravity(RPhysWorld* W, RPhysVec3 g3) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_gravity: world is null");
  std::lock_guard<std::mutex> g(W->mu);
  W->w.gravity = v(g3);
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_heightfield_f32(RPhysWorld* W, uint32_t nx, uint32_t nz, float cx, float cz, float ox, float oz,
                                          const float* h, uint32_t mat) {
  clear_err();
  if (!W || !h) return fail(RPHYS_ERR_NULL, "rphys_ext_set_heightfield_f32: null arg");
  if (nx == 0 || nz == 0) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_heightfield_f32: nx/nz == 0");
  if (!material_known(mat)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_heightfield_f32: unknown material");
  std::vector<float> hh(h, h + (size_t)nx * nz);
  std::lock_guard<std::mutex> g(W->mu);
  return set_hf(W, nx, nz, cx, cz, ox, oz, std::move(hh), mat);
}
RPhysResult rphys_ext_set_residual_mode(RPhysWorld* W, float tol, uint32_t max_sweeps) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_residual_mode: world is null");
  if (!std::isfinite(tol)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_residual_mode: tolerance not finite");
  std::lock_guard<std::mutex> g(W->mu);
  W->w.res_tol = tol; W->w.res_max = max_sweeps;
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_solve_order(RPhysWorld* W, uint32_t order) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_solve_order: world is null");
  if (order > RPHYS_ORDER_COLOURED) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_solve_order: unknown order");
  std::lock_guard<std::mutex> g(W->mu);
  W->w.coloured = order == RPHYS_ORDER_COLOURED;
  return RPHYS_OK;
}
// Launch shapes mean nothing on the CPU: checked like the CUDA library's, stored and returned.
RPhysResult rphys_ext_set_tuning(RPhysWorld* W, const RPhysTuning* t) {
  clear_err();
  if (!W || !t) return fail(RPHYS_ERR_NULL, "rphys_ext_set_tuning: null arg");
  auto in = [](uint32_t v, uint32_t a, uint32_t b, uint32_t c) { return v == a || v == b || v == c; };
  if (!((in(t->group_rows, 8, 16, 32) || in(t->group_rows, 64, 128, 128)) && in(t->packed_threads, 32, 64, 128) &&
        (t->island_threads == 32 || in(t->island_threads, 64, 128, 256))))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_tuning: unsupported launch shape");
  std::lock_guard<std::mutex> g(W->mu);
  W->tuning = *t;
  return RPHYS_OK;
}
RPhysResult rphys_ext_get_tuning(const RPhysWorld* Wc, RPhysTuning* out) {
  clear_err();
  if (!Wc || !out) return fail(RPHYS_ERR_NULL, "rphys_ext_get_tuning: null arg");
  *out = Wc->tuning;
  return RPHYS_OK;
}
RPhysResult rphys_ext_add_joints(RPhysWorld* W, const RPhysJointDesc* d, uint32_t n, uint32_t* out_first) {
  clear_err();
  if (out_first) *out_first = 0;
  if (!W || (!d && n) || !out_first) return fail(RPHYS_ERR_NULL, "rphys_ext_add_joints: null arg");
  std::lock_guard<std::mutex> g(W->mu);
  std::vector<std::pair<uint32_t, uint32_t>> ab(n);
  for (uint32_t i = 0; i < n; ++i) {
    if (d[i].kind > RPHYS_JOINT_D6 || (d[i].kind == RPHYS_JOINT_HINGE && d[i].hinge_axis > 2))
      return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_joints: bad kind or hinge axis");
    if (!fin_iso(d[i].frame_a) || !fin_iso(d[i].frame_b)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_joints: frame contains NaN/Inf");
    RPhysResult r = live_id(W, d[i].body_a, "rphys_ext_add_joints", &ab[i].first);
    if (r) return r;
    r = live_id(W, d[i].body_b, "rphys_ext_add_joints", &ab[i].second);
    if (r) return r;
    if (ab[i].first == ab[i].second) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_joints: body_a == body_b");
  }
  *out_first = (uint32_t)W->w.joints.size();
  for (uint32_t i = 0; i < n; ++i) {
    Iso fa{v(d[i].frame_a.pos), q(d[i].frame_a.rot)}, fb{v(d[i].frame_b.pos), q(d[i].frame_b.rot)};
    if (d[i].kind == RPHYS_JOINT_BALL) W->w.add_ball_joint(ab[i].first, ab[i].second, fa, fb);
    else if (d[i].kind == RPHYS_JOINT_HINGE) W->w.add_hinge_joint(ab[i].first, ab[i].second, fa, fb, d[i].hinge_axis);
    else W->w.add_d6_joint(ab[i].first, ab[i].second, fa, fb);
  }
  return RPHYS_OK;
}
RPhysResult rphys_ext_add_distance_joints(RPhysWorld* W, const RPhysDistanceJointDesc* d, uint32_t n,
                                          uint32_t* out_first) {
  clear_err();
  if (out_first) *out_first = 0;
  if (!W || (!d && n) || !out_first) return fail(RPHYS_ERR_NULL, "rphys_ext_add_distance_joints: null arg");
  std::lock_guard<std::mutex> g(W->mu);
  std::vector<std::pair<uint32_t, uint32_t>> ab(n);
  auto fin3 = [](RPhysVec3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); };
  for (uint32_t i = 0; i < n; ++i) {
    if (!fin3(d[i].anchor_a) || !fin3(d[i].anchor_b) || !std::isfinite(d[i].rest) ||
        !(std::isfinite(d[i].compliance) && d[i].compliance >= 0.0f) ||
        !(std::isfinite(d[i].damping) && d[i].damping >= 0.0f))
      return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_distance_joints: non-finite value or negative compliance / damping");
    RPhysResult r = live_id(W, d[i].body_a, "rphys_ext_add_distance_joints", &ab[i].first);
    if (r) return r;
    r = live_id(W, d[i].body_b, "rphys_ext_add_distance_joints", &ab[i].second);
    if (r) return r;
    if (ab[i].first == ab[i].second) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_distance_joints: body_a == body_b");
  }
  *out_first = (uint32_t)W->w.joints.size();
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t id = W->w.add_distance_joint_at(ab[i].first, v(d[i].anchor_a), ab[i].second, v(d[i].anchor_b), d[i].rest,
                                             d[i].compliance);
    W->w.set_distance_damping(id, d[i].damping);
  }
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_joint_limit(RPhysWorld* W, uint32_t joint, uint32_t angular, uint32_t axis, uint32_t enabled,
                                      float lo, float hi) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_joint_limit: world is null");
  std::lock_guard<std::mutex> g(W->mu);
  if (joint >= W->w.joints.size()) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_set_joint_limit: joint out of range");
  if (axis > 2) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_limit: axis > 2");
  if (enabled && !(std::isfinite(lo) && std::isfinite(hi) && lo <= hi))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_limit: limit must be finite with lo <= hi");
  W->w.set_d6_limit(joint, angular != 0, axis, enabled != 0, lo, hi);
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_joint_limits(RPhysWorld* W, const RPhysJointLimit* l, uint32_t n) {
  clear_err();
  if (!W || (!l && n)) return fail(RPHYS_ERR_NULL, "rphys_ext_set_joint_limits: null arg");
  std::lock_guard<std::mutex> g(W->mu);
  for (uint32_t i = 0; i < n; ++i) {
    if (l[i].joint >= W->w.joints.size()) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_set_joint_limits: joint out of range");
    if (l[i].axis > 2) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_limits: axis > 2");
    if (l[i].enabled && !(std::isfinite(l[i].lo) && std::isfinite(l[i].hi) && l[i].lo <= l[i].hi))
      return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_limits: limit must be finite with lo <= hi");
  }
  for (uint32_t i = 0; i < n; ++i) W->w.set_d6_limit(l[i].joint, l[i].angular != 0, l[i].axis, l[i].enabled != 0, l[i].lo, l[i].hi);
  return RPHYS_OK;
}
// Test hook: f32 values d in [0.8, 1] where the restated turned test 2 acos(d) < 0.5 and the
// threshold form d >= dstar disagree (the GPU evaluates the threshold form).
uint32_t rphys_oracle_turned_threshold_mismatches(uint32_t dstar_bits) {
  float dstar;
  std::memcpy(&dstar, &dstar_bits, 4);
  uint32_t bad = 0;
  for (float d = 0.8f; d <= 1.0f; d = std::nextafter(d, 2.0f))
    if ((2.0f * om::acosf_unit_rp(d) < 0.5f) != (d >= dstar)) bad++;
  return bad;
}
// Test hook: SHAKE_MAX_TURN.cos() as the oracle computes it (its bits; the GPU carries them as a
// constant).
uint32_t rphys_oracle_shake_max_turn_cos_bits() {
  float s, c;
  om::sincosf_rp(0.5f, &s, &c);
  uint32_t u;
  std::memcpy(&u, &c, 4);
  return u;
}
// Test hook: the distance-joint scenes of the reference's golden bit test
// (riftphys-world/tests/distance_bits_test.rs:11-48), built on the oracle World directly (no
// colliders, as World::add_body makes none): a 0.2 x 0.1 x 0.16 m box of density 500 swinging on a
// distance joint from a static pivot at (0, 5, 0), kind 0 rigid at its start length, kind 1 a
// spring (compliance 2e-3 m/N) at 0.8 of it; 3 s at hz. Returns the FNV-1a fold of the box's
// pose and velocity bits, the reference test's bits().
uint64_t rphys_oracle_distance_bits(uint32_t kind, float hz) {
  using namespace om;
  orc::World w(8);
  w.gravity = V3{0.0f, -9.81f, 0.0f};
  uint32_t pivot = w.add_body(Iso{V3{0.0f, 5.0f, 0.0f}, Q4{0, 0, 0, 1}}, V3{0, 0, 0}, V3{0, 0, 0}, 0.0f, V3{0, 0, 0}, false);
  const float he[3] = {0.1f, 0.05f, 0.08f};
  float im;
  V3 inertia;
  orc::mass_from_density(orc::SH_BOX, he, 500.0f, &im, &inertia);
  float sy, cy, sx, cx;
  sincosf_rp(0.3f * 0.5f, &sy, &cy);  // Quat::from_rotation_y(0.3)
  sincosf_rp(0.2f * 0.5f, &sx, &cx);  // Quat::from_rotation_x(0.2)
  Q4 rot = qmul(Q4{0.0f, sy, 0.0f, cy}, Q4{sx, 0.0f, 0.0f, cx});
  V3 start{0.7f, 4.3f, 0.2f};
  uint32_t b = w.add_body(Iso{start, rot}, V3{0.0f, 0.5f, 1.5f}, V3{0.4f, -1.0f, 2.0f}, im, inertia, true);
  w.sleep_allowed[b] = 0;
  float rest = len(sub(start, V3{0.0f, 5.0f, 0.0f}));
  if (kind == 0) w.add_distance_joint(pivot, b, rest, 0.0f);
  else w.add_distance_joint(pivot, b, rest * 0.8f, 2.0e-3f);
  const uint32_t n = (uint32_t)(3.0f * hz);
  for (uint32_t t = 0; t < n; ++t) w.step(1.0f / hz);
  uint64_t h = 0xcbf29ce484222325ull;
  const float x[13] = {w.pos[b].x, w.pos[b].y, w.pos[b].z, w.rot[b].x, w.rot[b].y, w.rot[b].z, w.rot[b].w,
                       w.lin[b].x, w.lin[b].y, w.lin[b].z, w.ang[b].x, w.ang[b].y, w.ang[b].z};
  for (float f : x) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    h = (h ^ (uint64_t)u) * 0x100000001b3ull;
  }
  return h;
}
RPhysResult rphys_ext_set_joint_axis(RPhysWorld* W, uint32_t joint, uint32_t angular, uint32_t axis, uint32_t enabled,
                                     float compliance) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_joint_axis: world is null");
  std::lock_guard<std::mutex> g(W->mu);
  if (joint >= W->w.joints.size()) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_set_joint_axis: joint out of range");
  if (axis > 2) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_axis: axis > 2");
  if (!(std::isfinite(compliance) && compliance >= 0.0f))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_axis: compliance must be finite and >= 0");
  W->w.set_d6_axis(joint, angular != 0, axis, enabled != 0, compliance);
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_joint_drive(RPhysWorld* W, uint32_t joint, uint32_t angular, uint32_t axis,
                                      const RPhysJointDrive* d) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_joint_drive: world is null");
  std::lock_guard<std::mutex> g(W->mu);
  if (joint >= W->w.joints.size()) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_set_joint_drive: joint out of range");
  if (axis > 2) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_drive: axis > 2");
  if (d && !(std::isfinite(d->target) && std::isfinite(d->kp) && std::isfinite(d->kd) && std::isfinite(d->max_impulse)))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_drive: non-finite drive value");
  if (d) W->w.set_d6_drive(joint, angular != 0, axis, true, d->target, d->kp, d->kd, d->max_impulse, d->vel_mode != 0);
  else W->w.set_d6_drive(joint, angular != 0, axis, false, 0.0f, 0.0f, 0.0f, 0.0f, false);
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_joint_damping(RPhysWorld* W, uint32_t joint, uint32_t angular, uint32_t axis, float damping,
                                        float friction) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_joint_damping: world is null");
  std::lock_guard<std::mutex> g(W->mu);
  if (joint >= W->w.joints.size()) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_set_joint_damping: joint out of range");
  if (axis > 2) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_damping: axis > 2");
  W->w.set_d6_damping(joint, angular != 0, axis, damping, friction);
  return RPHYS_OK;
}
RPhysResult rphys_ext_num_joints(const RPhysWorld* W, uint32_t* out) {
  clear_err();
  if (!W || !out) return fail(RPHYS_ERR_NULL, "rphys_ext_num_joints: null arg");
  *out = (uint32_t)W->w.joints.size();
  return RPHYS_OK;
}
RPhysResult rphys_ext_step_n(RPhysWorld* W, float dt, uint32_t n) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_step_n: world is null");
  if (!std::isfinite(dt) || dt < 0) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_step_n: bad dt");
  std::lock_guard<std::mutex> g(W->mu);
  for (uint32_t i = 0; i < n; ++i) W->w.step(dt);
  return RPHYS_OK;
}
RPhysResult rphys_ext_get_stats(const RPhysWorld* Wc, RPhysStepStats* o) {
  clear_err();
  if (!Wc || !o) return fail(RPHYS_ERR_NULL, "rphys_ext_get_stats: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  const Stats& s = W->w.stats;
  std::memset(o, 0, sizeof(*o));
  o->pairs = s.pairs; o->contacts = s.contacts; o->islands = s.islands; o->levels = s.levels;
  o->max_batch = s.max_batch; o->warm_matched = s.warm_matched; o->sweeps = s.sweeps;
  o->bounce_rows = s.bounce_rows; o->residual = s.residual;
  o->row_sweeps = s.row_sweeps; o->rows_scheduled = s.rows_scheduled;
  o->islands_capped = s.islands_capped;
  o->pred_used = s.pred_used;
  o->rows_capped = s.rows_capped;
  for (int k = 0; k < 6; ++k) o->res_hist[k] = s.res_hist[k];
  uint32_t we = 0;
  for (auto& kv : W->w.warm) we += (uint32_t)kv.second.size();
  o->warm_entries = we;
  o->sleeping = W->w.num_sleeping();
  return RPHYS_OK;
}
RPhysResult rphys_ext_get_pairs(const RPhysWorld* Wc, uint32_t* out, uint32_t cap, uint32_t* out_count) {
  clear_err();
  if (!Wc || !out_count) return fail(RPHYS_ERR_NULL, "rphys_ext_get_pairs: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  auto& p = W->w.last_pairs;
  *out_count = (uint32_t)p.size();
  if (!out) return RPHYS_OK;
  for (uint32_t i = 0; i < p.size() && i < cap; ++i) { out[2 * i] = p[i].first; out[2 * i + 1] = p[i].second; }
  return RPHYS_OK;
}
RPhysResult rphys_ext_get_contact_records(const RPhysWorld* Wc, RPhysContactRecord* out, uint32_t cap, uint32_t* out_count) {
  clear_err();
  if (!Wc || !out_count) return fail(RPHYS_ERR_NULL, "rphys_ext_get_contact_records: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  auto& cs = W->w.last_frame_contacts;
  *out_count = (uint32_t)cs.size();
  if (!out) return RPHYS_OK;
  for (uint32_t i = 0; i < cs.size() && i < cap; ++i) {
    const Contact& c = cs[i];
    RPhysContactRecord r;
    r.a_collider = c.a_collider; r.b_collider = c.b_collider;
    r.point = RPhysVec3{c.point.x, c.point.y, c.point.z};
    r.normal = RPhysVec3{c.normal.x, c.normal.y, c.normal.z};
    r.depth = c.depth; r.impulse = c.impulse;
    r.level = i < W->w.last_levels.size() ? W->w.last_levels[i] : 0xFFFFFFFFu;
    r.pad = 0;
    out[i] = r;
  }
  return RPHYS_OK;
}
RPhysResult rphys_ext_get_body_states(const RPhysWorld* Wc, uint32_t first, uint32_t count, float* out) {
  clear_err();
  if (!Wc || (!out && count)) return fail(RPHYS_ERR_NULL, "rphys_ext_get_body_states: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  std::lock_guard<std::mutex> g(W->mu);
  World& w = W->w;
  if ((uint64_t)first + count > w.num_bodies()) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_get_body_states: range out of bounds");
  for (uint32_t k = 0; k < count; ++k) {
    uint32_t i = first + k;
    float* o = out + 13 * (size_t)k;
    o[0] = w.pos[i].x; o[1] = w.pos[i].y; o[2] = w.pos[i].z;
    o[3] = w.rot[i].x; o[4] = w.rot[i].y; o[5] = w.rot[i].z; o[6] = w.rot[i].w;
    o[7] = w.lin[i].x; o[8] = w.lin[i].y; o[9] = w.lin[i].z;
    o[10] = w.ang[i].x; o[11] = w.ang[i].y; o[12] = w.ang[i].z;
  }
  return RPHYS_OK;
}

RPhysResult rphys_ext_profile_enable(RPhysWorld* W, uint32_t) { return W ? RPHYS_OK : RPHYS_ERR_NULL; }
RPhysResult rphys_ext_profile_read(const RPhysWorld* W, double*, uint64_t*, uint32_t, uint32_t* n) {
  if (!W || !n) return RPHYS_ERR_NULL;
  *n = 0;
  return RPHYS_OK;
}
const char* rphys_ext_profile_stage_name(uint32_t) { return nullptr; }
RPhysResult rphys_ext_stream_handle(const RPhysWorld* W, uint64_t* out) {
  if (!W || !out) return RPHYS_ERR_NULL;
  *out = 0;
  return RPHYS_OK;
}

RPhysResult rphys_ext_launch_count(uint64_t* out) {
  if (!out) return RPHYS_ERR_NULL;
  *out = 0;
  return RPHYS_OK;
}

// Oracle-only: CPU threads for the timed baseline (narrowphase and level batches, order-preserving).
RPhysResult rphys_oracle_set_threads(RPhysWorld* W, int threads) {
  if (!W) return RPHYS_ERR_NULL;
  std::lock_guard<std::mutex> g(W->mu);
  W->w.threads = threads < 1 ? 1 : threads;
  return RPHYS_OK;
}
// Oracle-only diagnostics: keep the worst solve island of each tick (rows and residual history).
RPhysResult rphys_oracle_diag_worst(RPhysWorld* W, int on) {
  if (!W) return RPHYS_ERR_NULL;
  std::lock_guard<std::mutex> g(W->mu);
  W->w.diag_worst = on != 0;
  return RPHYS_OK;
}
// Copies the last tick's worst island: up to cap_rows rows of 5 floats (body a, body b as bits,
// m_n, jn, the row's residual in the last sweep), up to cap_hist residuals.
RPhysResult rphys_oracle_diag_read(RPhysWorld* W, float* rows, uint32_t cap_rows, float* hist, uint32_t cap_hist,
                                   uint32_t* n_rows, uint32_t* n_hist) {
  if (!W || !n_rows || !n_hist) return RPHYS_ERR_NULL;
  std::lock_guard<std::mutex> g(W->mu);
  const World& w = W->w;
  *n_rows = (uint32_t)(w.diag_rows.size() / 5);
  *n_hist = (uint32_t)w.diag_hist.size();
  for (uint32_t k = 0; rows && k < 5 * std::min(cap_rows, *n_rows); ++k) rows[k] = w.diag_rows[k];
  for (uint32_t k = 0; hist && k < std::min(cap_hist, *n_hist); ++k) hist[k] = w.diag_hist[k];
  return RPHYS_OK;
}
// Oracle-only: BLAKE3 of a byte buffer (known-answer tests).
void rphys_oracle_blake3(const uint8_t* data, size_t n, uint8_t out[32]);

}  // extern "C"

#include "blake3_spec.h"
extern "C" void rphys_oracle_blake3(const uint8_t* data, size_t n, uint8_t out[32]) {
  b3::Hasher h;
  h.update(data, n);
  h.finalize(out);
}

// Oracle-only: collide_shapes on two posed shapes (narrowphase unit tests). shape: 0 sphere,
// 1 box, 2 capsule; dims as RPhysBodyDescEx; pose7 = pos xyz, rot xyzw. Writes up to 4 points as
// (position xyz, normal xyz, penetration) into out7x4; returns the point count (0: no contact).
extern "C" int rphys_oracle_collide(uint32_t sa, const float* da, const float* pa, uint32_t sb, const float* db,
                                    const float* pb, float cd, float* out) {
  Shape A{sa, da[0], da[1], da[2], V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}};
  Shape B{sb, db[0], db[1], db[2], V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}};
  Iso xa{V3{pa[0], pa[1], pa[2]}, Q4{pa[3], pa[4], pa[5], pa[6]}};
  Iso xb{V3{pb[0], pb[1], pb[2]}, Q4{pb[3], pb[4], pb[5], pb[6]}};
  Manifold m;
  if (!collide_shapes(A, xa, B, xb, cd, &m)) return 0;
  for (int k = 0; k < m.len; ++k) {
    float* o = out + 7 * k;
    o[0] = m.pts[k].position.x; o[1] = m.pts[k].position.y; o[2] = m.pts[k].position.z;
    o[3] = m.pts[k].normal.x; o[4] = m.pts[k].normal.y; o[5] = m.pts[k].normal.z;
    o[6] = m.pts[k].penetration;
  }
  return m.len;
}

// The learned warm start's model runs on the tensor cores only; the CPU restatement exports the
// symbols for the shared bindings and refuses (the tests check the model against numpy).
struct RPhysWarmModel { int unused; };
extern "C" {
RPhysWarmModel* rphys_ext_model_create(uint64_t) { fail(RPHYS_ERR_BAD_ARG, "model: GPU only"); return nullptr; }
void rphys_ext_model_destroy(RPhysWarmModel*) {}
uint32_t rphys_ext_model_num_params(void) { return 39312u; }
RPhysResult rphys_ext_model_get_weights(const RPhysWarmModel*, float*, uint32_t) { return fail(RPHYS_ERR_BAD_ARG, "model: GPU only"); }
RPhysResult rphys_ext_model_set_weights(RPhysWarmModel*, const float*, uint32_t) { return fail(RPHYS_ERR_BAD_ARG, "model: GPU only"); }
RPhysResult rphys_ext_model_predict(RPhysWarmModel*, const float*, uint32_t, float*) { return fail(RPHYS_ERR_BAD_ARG, "model: GPU only"); }
RPhysResult rphys_ext_model_predict_device(RPhysWarmModel*, const float*, uint32_t, float*, uint64_t) {
  return fail(RPHYS_ERR_BAD_ARG, "model: GPU only");
}
RPhysResult rphys_ext_model_gradients(RPhysWarmModel*, const float*, const float*, uint32_t, float*, float*) {
  return fail(RPHYS_ERR_BAD_ARG, "model: GPU only");
}
RPhysResult rphys_ext_model_train(RPhysWarmModel*, const float*, const float*, uint32_t, uint32_t, uint32_t, float, float*) {
  return fail(RPHYS_ERR_BAD_ARG, "model: GPU only");
}
}

// The learned warm start's model runs on the GPU; the restatement takes the predictions the GPU
// offered (rphys_ext_get_row_predictions) through rphys_oracle_set_predictions and makes the same
// per-row choice, so a learned-mode tick is checked bit for bit.
extern "C" {
RPhysResult rphys_ext_set_warm_model(RPhysWorld* W, RPhysWarmModel* M) {
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_warm_model: world is null");
  return M ? fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_warm_model: the restatement takes predictions, not a model") : RPHYS_OK;
}
RPhysResult rphys_ext_set_warm_policy(RPhysWorld* W, uint32_t) {
  return W ? RPHYS_OK : fail(RPHYS_ERR_NULL, "rphys_ext_set_warm_policy: world is null");
}
RPhysResult rphys_ext_set_feature_logging(RPhysWorld* W, uint32_t on) {
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_feature_logging: world is null");
  return on ? fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_feature_logging: GPU only") : RPHYS_OK;
}
RPhysResult rphys_ext_get_row_features(const RPhysWorld* W, float*, float*, uint32_t, uint32_t* n) {
  if (!W || !n) return fail(RPHYS_ERR_NULL, "rphys_ext_get_row_features: null arg");
  *n = 0;
  return RPHYS_OK;
}
RPhysResult rphys_ext_get_row_predictions(const RPhysWorld* W, float*, uint32_t, uint32_t* n) {
  if (!W || !n) return fail(RPHYS_ERR_NULL, "rphys_ext_get_row_predictions: null arg");
  *n = 0;
  return RPHYS_OK;
}
RPhysResult rphys_oracle_set_predictions(RPhysWorld* W, const float* pred4, uint32_t n_contacts) {
  if (!W || (!pred4 && n_contacts)) return fail(RPHYS_ERR_NULL, "rphys_oracle_set_predictions: null arg");
  std::lock_guard<std::mutex> g(W->mu);
  W->w.next_pred.assign(pred4, pred4 + 4 * (size_t)n_contacts);
  return RPHYS_OK;
}
}
