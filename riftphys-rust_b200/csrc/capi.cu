// capi.cu -- the drop-in boundary: the reference's C ABI v1 (crates/riftphys-ffi/src/lib.rs,
// riftphys_c.h) and the rphys_ext_ extensions, over the GPU world. Each call validates its
// arguments in the reference's order, clears and sets the thread-local error message, writes
// the deterministic default to out-params first, takes the world's mutex, and converts any C++
// or CUDA failure into RPHYS_ERR_INTERNAL (the reference's ffi_guard, lib.rs:97-106).
// step_ex synchronises before returning, so every getter sees the finished tick.
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <memory>
#include <mutex>
#include <string>

#include "../../include/rphys_ext.h"
#include "warm_model.h"
#include "world_gpu.h"

using rp::WorldGpu;
namespace rp {
extern unsigned long long g_launches;
}

static thread_local std::string g_err;
static thread_local bool g_has_err = false;
static void clear_err() { g_has_err = false; g_err.clear(); }
static RPhysResult fail(RPhysResult code, const std::string& m) { g_err = m; g_has_err = true; return code; }

struct RPhysWorld {
  std::mutex mu;
  std::unique_ptr<WorldGpu> w;
  uint32_t bodies_created = 0, colliders_created = 0, max_bodies, max_colliders;
  // contacts of the last tick, as the reference's last_frame_contacts (step.rs:384)
  RPhysWorld(uint32_t mb, uint32_t mc) : w(new WorldGpu(mb, mc)), max_bodies(mb), max_colliders(mc) {}
};
struct RPhysWorldSnapshot { rp::SnapshotGpu* s; };

template <class F>
static RPhysResult guard(const char* ctx, F f) {
  try {
    return f();
  } catch (const std::exception& e) {
    return fail(RPHYS_ERR_INTERNAL, std::string(ctx) + ": " + e.what());
  } catch (...) {
    return fail(RPHYS_ERR_INTERNAL, std::string(ctx) + ": internal failure");
  }
}
static bool fin3(const RPhysVec3& a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
static bool fin_iso(const RPhysIsometry& p) {
  return fin3(p.pos) && std::isfinite(p.rot.x) && std::isfinite(p.rot.y) && std::isfinite(p.rot.z) && std::isfinite(p.rot.w);
}
static bool fin_vel(const RPhysVelocity& a) { return fin3(a.lin) && fin3(a.ang); }
static bool fin_mat(const RPhysMaterial& m) {
  return std::isfinite(m.mu_static) && std::isfinite(m.mu_dynamic) && std::isfinite(m.restitution);
}
// checked_live_body_id (lib.rs:373-409)
static RPhysResult live_id(RPhysWorld* W, uint32_t id, const std::string& ctx, uint32_t* out) {
  if (id == 0) return fail(RPHYS_ERR_INVALID_ID, ctx + ": body_id == 0 (invalid)");
  if (id == RPHYS_TERRAIN_BODY_ID) return fail(RPHYS_ERR_INVALID_ID, ctx + ": body_id is terrain sentinel (not a real body)");
  uint32_t raw = id - 1;
  if (raw >= W->bodies_created) return fail(RPHYS_ERR_INVALID_ID, ctx + ": body_id out of range");
  if (!W->w->alive(raw)) return fail(RPHYS_ERR_INVALID_ID, ctx + ": body_id not found (removed)");
  *out = raw;
  return RPHYS_OK;
}
static void pose7(const RPhysIsometry& p, float o[7]) {
  o[0] = p.pos.x; o[1] = p.pos.y; o[2] = p.pos.z; o[3] = p.rot.x; o[4] = p.rot.y; o[5] = p.rot.z; o[6] = p.rot.w;
}
static void vel6(const RPhysVelocity& v, float o[6]) {
  o[0] = v.lin.x; o[1] = v.lin.y; o[2] = v.lin.z; o[3] = v.ang.x; o[4] = v.ang.y; o[5] = v.ang.z;
}
static RPhysResult add_one(RPhysWorld* W, const std::string& ctx, const RPhysIsometry& pose, const RPhysVelocity& vel,
                           uint32_t shape, const float dims[3], float density, bool dynamic, uint32_t mat, bool sleep_ok,
                           uint32_t* out) {
  if (W->bodies_created + 1ull > W->max_bodies) return fail(RPHYS_ERR_CAPACITY, ctx + ": body capacity exceeded");
  if (W->colliders_created + 1ull > W->max_colliders) return fail(RPHYS_ERR_CAPACITY, ctx + ": collider capacity exceeded");
  float im = 0, in[3] = {0, 0, 0};
  if (dynamic) rp::mass_from_density(shape, dims, density, &im, in);
  float p[7], v[6];
  pose7(pose, p); vel6(vel, v);
  uint32_t id = W->w->add_body(p, v, shape, dims, im, in, dynamic, mat, sleep_ok);
  if (id != W->bodies_created) return fail(RPHYS_ERR_INTERNAL, ctx + ": internal body id reuse/skip");
  W->bodies_created++;
  W->colliders_created++;
  *out = id + 1;
  return RPHYS_OK;
}
#define LOCK std::lock_guard<std::mutex> lk(W->mu)

extern "C" {

uint32_t rphys_get_abi_version(void) { return RPHYS_ABI_VERSION; }
const char* rphys_get_build_id(void) { return "riftphys_ffi-b200-0.1.0"; }
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
  try {
    return new RPhysWorld(max_bodies, max_colliders);
  } catch (const std::exception& e) {
    fail(RPHYS_ERR_INTERNAL, std::string("rphys_world_create: ") + e.what());
    return nullptr;
  }
}
void rphys_world_destroy(RPhysWorld* w) {
  try { delete w; } catch (...) {}
}
RPhysResult rphys_world_set_epoch(RPhysWorld* W, uint64_t e) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_world_set_epoch: world is null");
  LOCK; W->w->set_epoch(e); return RPHYS_OK;
}
RPhysResult rphys_world_set_rng_seed(RPhysWorld* W, uint64_t s) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_world_set_rng_seed: world is null");
  LOCK; W->w->set_rng_state(s | 1ull); return RPHYS_OK;  // XorShift64::new (rng.rs:7-9)
}

#define BODY_PRELUDE(NAME)                                                                                   \
  clear_err();                                                                                               \
  const std::string ctx = NAME;                                                                              \
  if (out) *out = 0;                                                                                         \
  if (!W || !d || !out) return fail(RPHYS_ERR_NULL, ctx + ": null arg");                                     \
  if (!fin_iso(d->pose)) return fail(RPHYS_ERR_BAD_ARG, ctx + ": pose contains NaN/Inf");                    \
  if (!fin_vel(d->vel)) return fail(RPHYS_ERR_BAD_ARG, ctx + ": vel contains NaN/Inf");                      \
  if (!fin_mat(d->material)) return fail(RPHYS_ERR_BAD_ARG, ctx + ": material contains NaN/Inf");
#define BODY_TYPE_CHECK                                                                                        \
  if (d->body_type > 1) return fail(RPHYS_ERR_BAD_ARG, ctx + ": invalid body_type");                           \
  if (d->body_type == 1 && !(std::isfinite(d->mass) && d->mass > 0))                                           \
    return fail(RPHYS_ERR_BAD_ARG, ctx + ": dynamic body mass must be finite and > 0");

// Dynamic FFI bodies get MaterialId::Default's density, 1500 kg/m^3, whatever the caller's mass
// (lib.rs:724-728; materials.rs:362), and keep material Default (mat_from_ffi, lib.rs:544-557).
RPhysResult rphys_add_capsule_body(RPhysWorld* W, const RPhysCapsuleBodyDesc* d, uint32_t* out) {
  BODY_PRELUDE("rphys_add_capsule_body")
  if (!(std::isfinite(d->radius) && d->radius > 0)) return fail(RPHYS_ERR_BAD_ARG, ctx + ": radius must be finite and > 0");
  if (!(std::isfinite(d->half_height) && d->half_height >= 0)) return fail(RPHYS_ERR_BAD_ARG, ctx + ": half_height must be finite and >= 0");
  BODY_TYPE_CHECK
  return guard(ctx.c_str(), [&]() {
    LOCK;
    float dims[3] = {d->radius, d->half_height, 0};
    return add_one(W, ctx, d->pose, d->vel, RPHYS_SHAPE_CAPSULE, dims, 1500.0f, d->body_type == 1, 0, true, out);
  });
}
RPhysResult rphys_add_box_body(RPhysWorld* W, const RPhysBoxBodyDesc* d, uint32_t* out) {
  BODY_PRELUDE("rphys_add_box_body")
  if (!(std::isfinite(d->hx) && d->hx > 0)) return fail(RPHYS_ERR_BAD_ARG, ctx + ": hx must be finite and > 0");
  if (!(std::isfinite(d->hy) && d->hy > 0)) return fail(RPHYS_ERR_BAD_ARG, ctx + ": hy must be finite and > 0");
  if (!(std::isfinite(d->hz) && d->hz > 0)) return fail(RPHYS_ERR_BAD_ARG, ctx + ": hz must be finite and > 0");
  BODY_TYPE_CHECK
  return guard(ctx.c_str(), [&]() {
    LOCK;
    float dims[3] = {d->hx, d->hy, d->hz};
    return add_one(W, ctx, d->pose, d->vel, RPHYS_SHAPE_BOX, dims, 1500.0f, d->body_type == 1, 0, true, out);
  });
}
RPhysResult rphys_add_sphere_body(RPhysWorld* W, const RPhysSphereBodyDesc* d, uint32_t* out) {
  BODY_PRELUDE("rphys_add_sphere_body")
  if (!(std::isfinite(d->radius) && d->radius > 0)) return fail(RPHYS_ERR_BAD_ARG, ctx + ": radius must be finite and > 0");
  BODY_TYPE_CHECK
  return guard(ctx.c_str(), [&]() {
    LOCK;
    float dims[3] = {d->radius, 0, 0};
    return add_one(W, ctx, d->pose, d->vel, RPHYS_SHAPE_SPHERE, dims, 1500.0f, d->body_type == 1, 0, true, out);
  });
}
RPhysResult rphys_body_remove(RPhysWorld* W, uint32_t id) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_body_remove: world is null");
  return guard("rphys_body_remove", [&]() {
    LOCK;
    uint32_t b;
    RPhysResult r = live_id(W, id, "rphys_body_remove", &b);
    if (r) return r;
    if (!W->w->remove_body(b)) return fail(RPHYS_ERR_INTERNAL, "rphys_body_remove: internal remove failed");
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_body_get_pose(const RPhysWorld* Wc, uint32_t id, RPhysIsometry* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_body_get_pose: out_pose is null");
  *out = RPhysIsometry{{0, 0, 0}, {0, 0, 0, 1}};
  if (!Wc) return fail(RPHYS_ERR_NULL, "rphys_body_get_pose: world is null");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_body_get_pose", [&]() {
    LOCK;
    uint32_t b;
    RPhysResult r = live_id(W, id, "rphys_body_get_pose", &b);
    if (r) return r;
    float p[7];
    W->w->get_body_pose(b, p);
    *out = RPhysIsometry{{p[0], p[1], p[2]}, {p[3], p[4], p[5], p[6]}};
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_body_set_pose(RPhysWorld* W, uint32_t id, const RPhysIsometry* p) {
  clear_err();
  if (!W || !p) return fail(RPHYS_ERR_NULL, "rphys_body_set_pose: null arg");
  if (!fin_iso(*p)) return fail(RPHYS_ERR_BAD_ARG, "rphys_body_set_pose: pose contains NaN/Inf");
  return guard("rphys_body_set_pose", [&]() {
    LOCK;
    uint32_t b;
    RPhysResult r = live_id(W, id, "rphys_body_set_pose", &b);
    if (r) return r;
    float q[7];
    pose7(*p, q);
    W->w->set_body_pose(b, q);
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_body_get_velocity(const RPhysWorld* Wc, uint32_t id, RPhysVelocity* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_body_get_velocity: out_vel is null");
  *out = RPhysVelocity{{0, 0, 0}, {0, 0, 0}};
  if (!Wc) return fail(RPHYS_ERR_NULL, "rphys_body_get_velocity: world is null");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_body_get_velocity", [&]() {
    LOCK;
    uint32_t b;
    RPhysResult r = live_id(W, id, "rphys_body_get_velocity", &b);
    if (r) return r;
    float v[6];
    W->w->get_body_vel(b, v);
    *out = RPhysVelocity{{v[0], v[1], v[2]}, {v[3], v[4], v[5]}};
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_body_set_velocity(RPhysWorld* W, uint32_t id, const RPhysVelocity* vel) {
  clear_err();
  if (!W || !vel) return fail(RPHYS_ERR_NULL, "rphys_body_set_velocity: null arg");
  if (!fin_vel(*vel)) return fail(RPHYS_ERR_BAD_ARG, "rphys_body_set_velocity: velocity contains NaN/Inf");
  return guard("rphys_body_set_velocity", [&]() {
    LOCK;
    uint32_t b;
    RPhysResult r = live_id(W, id, "rphys_body_set_velocity", &b);
    if (r) return r;
    float v[6];
    vel6(*vel, v);
    W->w->set_body_vel(b, v);
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_body_apply_impulse(RPhysWorld* W, uint32_t id, RPhysVec3 imp) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_body_apply_impulse: world is null");
  if (!fin3(imp)) return fail(RPHYS_ERR_BAD_ARG, "rphys_body_apply_impulse: impulse contains NaN/Inf");
  return guard("rphys_body_apply_impulse", [&]() {
    LOCK;
    uint32_t b;
    RPhysResult r = live_id(W, id, "rphys_body_apply_impulse", &b);
    if (r) return r;
    float j[3] = {imp.x, imp.y, imp.z};
    W->w->apply_impulse(b, j);
    return (RPhysResult)RPHYS_OK;
  });
}

RPhysResult rphys_world_step_ex(RPhysWorld* W, const RPhysStepParams* p) {
  clear_err();
  if (!W || !p) return fail(RPHYS_ERR_NULL, "rphys_world_step_ex: null arg");
  if (p->size_bytes < sizeof(RPhysStepParams)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_step_ex: size_bytes too small");
  if (!std::isfinite(p->dt)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_step_ex: dt is not finite");
  if (p->dt < 0) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_step_ex: dt is negative");
  if (p->substeps == 0) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_step_ex: substeps == 0");
  return guard("rphys_world_step_ex", [&]() {
    LOCK;
    float sub = p->dt / (float)p->substeps;
    if (!std::isfinite(sub)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_step_ex: sub_dt is not finite");
    for (uint32_t i = 0; i < p->substeps; ++i) W->w->step(sub);  // solver_iters and flags ignored (lib.rs:1147-1148)
    W->w->synchronize();
    return (RPhysResult)RPHYS_OK;
  });
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
  LOCK;
  *out = W->w->tick();
  return RPHYS_OK;
}
RPhysResult rphys_world_num_bodies(const RPhysWorld* Wc, uint32_t* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_world_num_bodies: out_num is null");
  *out = 0;
  if (!Wc) return fail(RPHYS_ERR_NULL, "rphys_world_num_bodies: world is null");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  LOCK;
  *out = W->w->num_bodies();
  return RPHYS_OK;
}
RPhysResult rphys_world_get_step_hash(const RPhysWorld* Wc, RPhysHash32* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_world_get_step_hash: out_hash is null");
  std::memset(out, 0, sizeof(*out));
  if (!Wc) return fail(RPHYS_ERR_NULL, "rphys_world_get_step_hash: world is null");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_world_get_step_hash", [&]() {
    LOCK;
    W->w->step_hash(out->bytes);
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_world_step_hash_noalloc(const RPhysWorld* Wc, RPhysHash32* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_ext_world_step_hash_noalloc: out_hash is null");
  std::memset(out, 0, sizeof(*out));
  if (!Wc) return fail(RPHYS_ERR_NULL, "rphys_ext_world_step_hash_noalloc: world is null");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_ext_world_step_hash_noalloc", [&]() {
    LOCK;
    try {
      W->w->step_hash_noalloc(out->bytes);
    } catch (const std::length_error& e) {
      return fail(RPHYS_ERR_CAPACITY, std::string("rphys_ext_world_step_hash_noalloc: ") + e.what());
    }
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_world_step_and_hash(RPhysWorld* W, float dt, RPhysHash32* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_world_step_and_hash: out_hash is null");
  std::memset(out, 0, sizeof(*out));
  RPhysResult r = rphys_world_step(W, dt);
  if (r) return r;
  return rphys_world_get_step_hash(W, out);
}

// HeightField::from_heights (terrain.rs:24-50): cell sizes and heights quantised to 1e-6.
static RPhysResult set_hf(RPhysWorld* W, uint32_t nx, uint32_t nz, float cx, float cz, float ox, float oz,
                          std::vector<float> h, uint32_t mat) {
  float sx = (std::isfinite(cx) && cx > 0) ? rp::q6(cx) : 1.0f;
  float sz = (std::isfinite(cz) && cz > 0) ? rp::q6(cz) : 1.0f;
  float mn = INFINITY, mx = -INFINITY;
  for (auto& x : h) {
    float v = std::isfinite(x) ? x : 0.0f;
    x = rp::q6(v);
    mn = rp::rmin(mn, x);
    mx = rp::rmax(mx, x);
  }
  W->w->set_heightfield(nx, nz, sx, sz, ox, oz, h, rp::q6(mn), rp::q6(mx), mat);
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
  return guard("rphys_world_set_heightfield_i16", [&]() {
    LOCK;
    return set_hf(W, d->width, d->height, d->cell_size_x, d->cell_size_z, ox, oz, std::move(h), 4);
  });
}
RPhysResult rphys_world_set_heightfield_raw32_square(RPhysWorld* W, const uint8_t* bytes, uint32_t n, float wx, float wz,
                                                     float ox, float oz, float yoff) {
  clear_err();
  if (!W || !bytes) return fail(RPHYS_ERR_NULL, "rphys_world_set_heightfield_raw32_square: null arg");
  if (n < 4) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_set_heightfield_raw32_square: bytes_len too small to form a grid");
  size_t cnt = n / 4;
  size_t dim = (size_t)std::sqrt((double)cnt);
  if (dim * dim != cnt) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_set_heightfield_raw32_square: byte length is not a square number of f32s");
  float cx = wx / rp::rmax((float)dim - 1.0f, 1.0f), cz = wz / rp::rmax((float)dim - 1.0f, 1.0f);
  std::vector<float> h(cnt);
  for (size_t i = 0; i < cnt; ++i) { float x; std::memcpy(&x, bytes + 4 * i, 4); h[i] = x + yoff; }
  return guard("rphys_world_set_heightfield_raw32_square", [&]() {
    LOCK;
    return set_hf(W, (uint32_t)dim, (uint32_t)dim, cx, cz, ox, oz, std::move(h), 4);
  });
}
RPhysResult rphys_world_clear_heightfield(RPhysWorld* W) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_world_clear_heightfield: world is null");
  LOCK;
  W->w->clear_heightfield();
  return RPHYS_OK;
}
RPhysResult rphys_world_get_contacts(const RPhysWorld* Wc, RPhysContactEvent* out, uint32_t cap, uint32_t* out_count) {
  clear_err();
  if (!Wc || !out_count) return fail(RPHYS_ERR_NULL, "rphys_world_get_contacts: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_world_get_contacts", [&]() {
    LOCK;
    std::vector<WorldGpu::ContactOut> cs;
    W->w->get_contacts(cs);
    *out_count = (uint32_t)cs.size();
    if (!out) return (RPhysResult)RPHYS_OK;
    uint32_t n = (uint32_t)cs.size() < cap ? (uint32_t)cs.size() : cap;
    for (uint32_t i = 0; i < n; ++i) {
      const auto& c = cs[i];
      RPhysContactEvent e;
      e.body_id_a = W->w->body_of_collider(c.a) + 1;
      e.body_id_b = c.b == 0xFFFFFFFFu ? RPHYS_TERRAIN_BODY_ID : W->w->body_of_collider(c.b) + 1;
      e.position = RPhysVec3{c.p[0], c.p[1], c.p[2]};
      e.normal = RPhysVec3{c.n[0], c.n[1], c.n[2]};
      e.impulse = c.impulse;
      out[i] = e;
    }
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_pack_snapshot(RPhysWorld* W, uint64_t tick, uint64_t epoch, uint8_t* out, uint64_t out_cap,
                                    uint64_t* out_bytes, uint32_t* out_chunks) {
  clear_err();
  if (out_bytes) *out_bytes = 0;
  if (out_chunks) *out_chunks = 0;
  if (!W || !out_bytes || !out_chunks) return fail(RPHYS_ERR_NULL, "rphys_ext_pack_snapshot: null arg");
  return guard("rphys_ext_pack_snapshot", [&]() {
    LOCK;
    size_t bytes = 0;
    uint32_t chunks = 0;
    W->w->pack_snapshot(tick, epoch, nullptr, 0, &bytes, &chunks);
    *out_bytes = bytes;
    *out_chunks = chunks;
    if (!out) return (RPhysResult)RPHYS_OK;
    if (out_cap < bytes) return fail(RPHYS_ERR_CAPACITY, "rphys_ext_pack_snapshot: buffer smaller than the snapshot");
    W->w->pack_snapshot(tick, epoch, out, (size_t)out_cap, &bytes, &chunks);
    return (RPhysResult)RPHYS_OK;
  });
}
// lib.rs:470-479
static void write_raycast_miss(RPhysRayHit* h) {
  h->hit = RPHYS_FALSE;
  h->body_id = RPHYS_INVALID_BODY_ID;
  h->fraction = 1.0f;
  h->point = RPhysVec3{0.0f, 0.0f, 0.0f};
  h->normal = RPhysVec3{0.0f, 1.0f, 0.0f};
}
// The checks and the direction normalisation of rphys_world_raycast (lib.rs:1286-1322) and of
// World::raycast (queries.rs:51-56); *cast = 1 when the ray is cast (ray8 filled), 0 for a miss.
static RPhysResult ray_prepare(RPhysWorld* W, const RPhysRayQuery& q, const char* ctx, float ray8[8], int* cast) {
  *cast = 0;
  auto fin3 = [](RPhysVec3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); };
  if (!fin3(q.origin)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": origin contains NaN/Inf");
  if (!fin3(q.dir)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": dir contains NaN/Inf");
  if (!std::isfinite(q.max_distance)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": max_distance is not finite");
  uint32_t ignore = 0xFFFFFFFFu;
  if (q.ignore_body != 0) {
    RPhysResult r = live_id(W, q.ignore_body, std::string(ctx) + ".ignore_body", &ignore);
    if (r) return r;
  }
  if (q.max_distance <= 0.0f) return RPHYS_OK;
  const float len2 = (q.dir.x * q.dir.x + q.dir.y * q.dir.y) + q.dir.z * q.dir.z;
  if (!std::isfinite(len2)) return fail(RPHYS_ERR_BAD_ARG, std::string(ctx) + ": dir length overflow/invalid");
  if (len2 <= 1.0e-20f) return RPHYS_OK;
  const float l = std::sqrt(len2);
  float dx = q.dir.x / l, dy = q.dir.y / l, dz = q.dir.z / l;
  const float len = std::sqrt((dx * dx + dy * dy) + dz * dz);  // World::raycast normalises again
  if (!std::isfinite(len) || len < 1.0e-12f) return RPHYS_OK;
  dx /= len; dy /= len; dz /= len;
  ray8[0] = q.origin.x; ray8[1] = q.origin.y; ray8[2] = q.origin.z;
  ray8[3] = dx; ray8[4] = dy; ray8[5] = dz;
  ray8[6] = q.max_distance;
  std::memcpy(ray8 + 7, &ignore, 4);
  *cast = 1;
  return RPHYS_OK;
}
static void ray_result(const float4& pt, const float4& n, RPhysRayHit* h) {
  uint32_t code;
  std::memcpy(&code, &pt.w, 4);
  if (code == 0) { write_raycast_miss(h); return; }
  h->hit = RPHYS_TRUE;
  h->body_id = code;  // id + 1, or RPHYS_TERRAIN_BODY_ID
  h->fraction = n.w;
  h->point = RPhysVec3{pt.x, pt.y, pt.z};
  h->normal = RPhysVec3{n.x, n.y, n.z};
}
RPhysResult rphys_world_raycast(const RPhysWorld* Wc, const RPhysRayQuery* q, RPhysRayHit* out) {
  clear_err();
  if (out) write_raycast_miss(out);
  if (!Wc || !q || !out) return fail(RPHYS_ERR_NULL, "rphys_world_raycast: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_world_raycast", [&]() {
    LOCK;
    float ray8[8];
    int cast = 0;
    RPhysResult r = ray_prepare(W, *q, "rphys_world_raycast", ray8, &cast);
    if (r || !cast) return r;
    float4 pt, n;
    W->w->raycast_batch(1, ray8, &pt, &n);
    ray_result(pt, n, out);
    return (RPhysResult)RPHYS_OK;
  });
}
static RPhysResult raycast_many(const RPhysWorld* Wc, const RPhysRayQuery* q, uint32_t n, RPhysRayHit* out, const char* ctx,
                                bool exact) {
  clear_err();
  if (!Wc || ((!q || !out) && n)) return fail(RPHYS_ERR_NULL, std::string(ctx) + ": null arg");
  for (uint32_t i = 0; i < n; ++i) write_raycast_miss(out + i);
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard(ctx, [&]() {
    LOCK;
    std::vector<float> rays;
    std::vector<uint32_t> which;
    rays.reserve(8 * (size_t)n);
    for (uint32_t i = 0; i < n; ++i) {
      float ray8[8];
      int cast = 0;
      RPhysResult r = ray_prepare(W, q[i], ctx, ray8, &cast);
      if (r) return r;
      if (cast) { rays.insert(rays.end(), ray8, ray8 + 8); which.push_back(i); }
    }
    const uint32_t m = (uint32_t)which.size();
    if (!m) return (RPhysResult)RPHYS_OK;
    std::vector<float4> pt(m), nn(m);
    W->w->raycast_batch(m, rays.data(), pt.data(), nn.data(), exact);
    for (uint32_t k = 0; k < m; ++k) ray_result(pt[k], nn[k], out + which[k]);
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_raycast_batch(const RPhysWorld* Wc, const RPhysRayQuery* q, uint32_t n, RPhysRayHit* out) {
  return raycast_many(Wc, q, n, out, "rphys_ext_raycast_batch", false);
}
// World::raycast_exact (queries.rs:18-48) for n rays, checked and normalised as rphys_world_raycast
RPhysResult rphys_ext_raycast_exact_batch(const RPhysWorld* Wc, const RPhysRayQuery* q, uint32_t n, RPhysRayHit* out) {
  return raycast_many(Wc, q, n, out, "rphys_ext_raycast_exact_batch", true);
}
// lib.rs:482-492
static void write_sweep_miss(RPhysCapsuleSweepHit* h) {
  h->hit = RPHYS_FALSE;
  h->body_id = RPHYS_INVALID_BODY_ID;
  h->fraction = 1.0f;
  h->started_overlapping = RPHYS_FALSE;
  h->point = RPhysVec3{0.0f, 0.0f, 0.0f};
  h->normal = RPhysVec3{0.0f, 1.0f, 0.0f};
}
RPhysResult rphys_world_capsule_sweep(const RPhysWorld* Wc, const RPhysCapsuleSweepQuery* q, RPhysCapsuleSweepHit* out) {
  clear_err();
  if (out) write_sweep_miss(out);
  if (!Wc || !q || !out) return fail(RPHYS_ERR_NULL, "rphys_world_capsule_sweep: null arg");
  auto fin3 = [](RPhysVec3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); };
  if (!fin3(q->from)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_capsule_sweep: from contains NaN/Inf");
  if (!fin3(q->to)) return fail(RPHYS_ERR_BAD_ARG, "rphys_world_capsule_sweep: to contains NaN/Inf");
  if (!(std::isfinite(q->radius) && q->radius > 0.0f))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_world_capsule_sweep: radius must be finite and > 0");
  if (!(std::isfinite(q->half_height) && q->half_height >= 0.0f))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_world_capsule_sweep: half_height must be finite and >= 0");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_world_capsule_sweep", [&]() {
    LOCK;
    uint32_t ignore = 0xFFFFFFFFu;
    if (q->ignore_body != 0) {
      RPhysResult r = live_id(W, q->ignore_body, "rphys_world_capsule_sweep.ignore_body", &ignore);
      if (r) return r;
    }
    float q12[12] = {q->from.x, q->from.y, q->from.z, q->to.x, q->to.y, q->to.z, q->radius, q->half_height, 0, 0, 0, 0};
    std::memcpy(q12 + 8, &ignore, 4);
    float4 pt, n;
    W->w->sweep_batch(1, q12, &pt, &n);
    uint32_t code;
    std::memcpy(&code, &pt.w, 4);
    if (code == 0) return (RPhysResult)RPHYS_OK;
    const bool overlap = n.w == 0.0f && std::signbit(n.w);
    out->hit = RPHYS_TRUE;
    out->body_id = code;
    out->fraction = overlap ? 0.0f : n.w;
    out->started_overlapping = overlap ? RPHYS_TRUE : RPHYS_FALSE;
    out->point = RPhysVec3{pt.x, pt.y, pt.z};
    out->normal = RPhysVec3{n.x, n.y, n.z};
    return (RPhysResult)RPHYS_OK;
  });
}
// rphys_add_player (lib.rs:1580-1627): the desc checked, then one body and one collider of
// capacity; World::add_player's body and capsule, the desc's size and speed on the controller.
RPhysResult rphys_add_player(RPhysWorld* W, const RPhysPlayerDesc* d, uint32_t* out) {
  clear_err();
  if (out) *out = 0xFFFFFFFFu;
  if (!W || !d || !out) return fail(RPHYS_ERR_NULL, "rphys_add_player: null arg");
  if (!fin_iso(d->start_pose)) return fail(RPHYS_ERR_BAD_ARG, "rphys_add_player: pose contains NaN/Inf");
  if (!(std::isfinite(d->radius) && d->radius > 0.0f)) return fail(RPHYS_ERR_BAD_ARG, "rphys_add_player: radius must be > 0");
  if (!(std::isfinite(d->height) && d->height > 0.0f)) return fail(RPHYS_ERR_BAD_ARG, "rphys_add_player: height must be > 0");
  return guard("rphys_add_player", [&]() {
    LOCK;
    if (W->bodies_created + 1ull > W->max_bodies) return fail(RPHYS_ERR_CAPACITY, "rphys_add_player: body capacity exceeded");
    if (W->colliders_created + 1ull > W->max_colliders)
      return fail(RPHYS_ERR_CAPACITY, "rphys_add_player: collider capacity exceeded");
    float p[7];
    pose7(d->start_pose, p);
    const uint32_t idx = W->w->add_player(p, d->radius, d->height, d->speed);
    W->bodies_created++;
    W->colliders_created++;
    *out = idx;
    return (RPhysResult)RPHYS_OK;
  });
}
// rphys_player_get_pose (lib.rs:1629-1666): identity and false written first
RPhysResult rphys_player_get_pose(const RPhysWorld* Wc, uint32_t idx, RPhysIsometry* out, RPhysBool* grounded) {
  clear_err();
  if (out) *out = RPhysIsometry{RPhysVec3{0, 0, 0}, RPhysQuat{0, 0, 0, 1}};
  if (grounded) *grounded = RPHYS_FALSE;
  if (!Wc || !out) return RPHYS_ERR_NULL;
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_player_get_pose", [&]() {
    LOCK;
    if (idx >= W->w->num_players()) return fail(RPHYS_ERR_BAD_ARG, "rphys_player_get_pose: player_idx out of bounds");
    float p[7];
    bool g = false;
    W->w->get_player(idx, p, &g);
    *out = RPhysIsometry{RPhysVec3{p[0], p[1], p[2]}, RPhysQuat{p[3], p[4], p[5], p[6]}};
    if (grounded) *grounded = g ? RPHYS_TRUE : RPHYS_FALSE;
    return (RPhysResult)RPHYS_OK;
  });
}
// rphys_player_set_input (lib.rs:1668-1693)
RPhysResult rphys_player_set_input(RPhysWorld* W, uint32_t idx, RPhysVec3 dir) {
  clear_err();
  if (!W) return RPHYS_ERR_NULL;
  if (!fin3(dir)) return fail(RPHYS_ERR_BAD_ARG, "rphys_player_set_input: move_dir NaN/Inf");
  return guard("rphys_player_set_input", [&]() {
    LOCK;
    if (idx >= W->w->num_players()) return fail(RPHYS_ERR_BAD_ARG, "rphys_player_set_input: player_idx out of bounds");
    const float v3[3] = {dir.x, dir.y, dir.z};
    W->w->set_player_input(idx, v3);
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysWorldSnapshot* rphys_world_snapshot_create(const RPhysWorld* Wc) {
  clear_err();
  if (!Wc) { fail(RPHYS_ERR_NULL, "rphys_world_snapshot_create: world is null"); return nullptr; }
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  try {
    LOCK;
    return new RPhysWorldSnapshot{W->w->snapshot_create()};
  } catch (const std::exception& e) {
    fail(RPHYS_ERR_INTERNAL, std::string("rphys_world_snapshot_create: ") + e.what());
    return nullptr;
  }
}
RPhysResult rphys_world_snapshot_restore(RPhysWorld* W, const RPhysWorldSnapshot* s) {
  clear_err();
  if (!W || !s) return fail(RPHYS_ERR_NULL, "rphys_world_snapshot_restore: null arg");
  return guard("rphys_world_snapshot_restore", [&]() {
    LOCK;
    W->w->snapshot_restore(s->s);
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_snapshot_restore_exact(RPhysWorld* W, const RPhysWorldSnapshot* s) {
  clear_err();
  if (!W || !s) return fail(RPHYS_ERR_NULL, "rphys_ext_snapshot_restore_exact: null arg");
  return guard("rphys_ext_snapshot_restore_exact", [&]() {
    LOCK;
    if (s->s->nb != W->w->num_bodies())
      return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_snapshot_restore_exact: bodies were added since the snapshot");
    W->w->snapshot_restore_exact(s->s);
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_state_export(const RPhysWorld* Wc, uint8_t* out, uint64_t out_cap, uint64_t* out_bytes) {
  clear_err();
  if (!Wc || !out_bytes) return fail(RPHYS_ERR_NULL, "rphys_ext_state_export: null arg");
  *out_bytes = 0;
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_ext_state_export", [&]() {
    LOCK;
    if (W->w->num_players()) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_state_export: a world with players has no state blob");
    uint64_t n = W->w->state_bytes();
    *out_bytes = n;
    if (!out) return (RPhysResult)RPHYS_OK;
    if (out_cap < n) return fail(RPHYS_ERR_CAPACITY, "rphys_ext_state_export: buffer smaller than the state");
    W->w->state_export(out);
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_state_import(RPhysWorld* W, const uint8_t* in, uint64_t bytes) {
  clear_err();
  if (!W || !in) return fail(RPHYS_ERR_NULL, "rphys_ext_state_import: null arg");
  return guard("rphys_ext_state_import", [&]() {
    LOCK;
    try {
      W->w->state_import(in, bytes);
    } catch (const std::invalid_argument& e) {
      return fail(RPHYS_ERR_BAD_ARG, std::string("rphys_ext_state_import: ") + e.what());
    }
    return (RPhysResult)RPHYS_OK;
  });
}
void rphys_world_snapshot_free(RPhysWorldSnapshot* s) {
  if (!s) return;
  try { WorldGpu::snapshot_free(s->s); } catch (...) {}
  delete s;
}

// ---------------------------------------------------------------- extensions
// Validates and adds n bodies (one collider each) in one upload; shared by rphys_ext_add_bodies
// and rphys_ext_batch_add_world (which first opens a new world).
static RPhysResult add_bodies_impl(RPhysWorld* W, const RPhysBodyDescEx* d, uint32_t n, uint32_t* out_first,
                                   const char* ctx, bool new_world, uint32_t* out_world) {
  const std::string c = ctx;
  for (uint32_t i = 0; i < n; ++i) {
    const RPhysBodyDescEx& e = d[i];
    if (!fin_iso(e.pose) || !fin_vel(e.vel)) return fail(RPHYS_ERR_BAD_ARG, c + ": pose/vel contains NaN/Inf");
    if (e.shape > 2 || e.body_type > 1 || !rp::material_known(e.material_id))
      return fail(RPHYS_ERR_BAD_ARG, c + ": bad shape/body_type/material");
    int nd = e.shape == 0 ? 1 : (e.shape == 1 ? 3 : 1);
    for (int k = 0; k < nd; ++k)
      if (!(std::isfinite(e.dims[k]) && e.dims[k] > 0)) return fail(RPHYS_ERR_BAD_ARG, c + ": dims must be finite and > 0");
    if (e.shape == 2 && !(std::isfinite(e.dims[1]) && e.dims[1] >= 0))
      return fail(RPHYS_ERR_BAD_ARG, c + ": half_height must be finite and >= 0");
    if (e.body_type == 1 && !(std::isfinite(e.density) && e.density > 0))
      return fail(RPHYS_ERR_BAD_ARG, c + ": density must be finite and > 0");
  }
  return guard(ctx, [&]() {
    LOCK;
    if ((uint64_t)W->bodies_created + n > W->max_bodies) return fail(RPHYS_ERR_CAPACITY, c + ": body capacity exceeded");
    if ((uint64_t)W->colliders_created + n > W->max_colliders) return fail(RPHYS_ERR_CAPACITY, c + ": collider capacity exceeded");
    if (new_world) {
      if (n == 0) return fail(RPHYS_ERR_BAD_ARG, c + ": a world needs at least one body");
      if (!W->w->batched() && W->w->num_bodies() > 0)
        return fail(RPHYS_ERR_BAD_ARG, c + ": a batch starts on an empty world");
      W->w->begin_world();
      if (out_world) *out_world = W->w->num_worlds() - 1;
    }
    if (n == 0) return (RPhysResult)RPHYS_OK;
    std::vector<float> p7(7 * (size_t)n), v6(6 * (size_t)n), dims(3 * (size_t)n), im(n), in3(3 * (size_t)n);
    std::vector<uint32_t> sh(n), mat(n);
    std::vector<uint8_t> dyn(n), sok(n);
    for (uint32_t i = 0; i < n; ++i) {
      const RPhysBodyDescEx& e = d[i];
      pose7(e.pose, &p7[7 * (size_t)i]);
      vel6(e.vel, &v6[6 * (size_t)i]);
      float dd[3] = {e.dims[0], e.shape == 0 ? 0.0f : e.dims[1], e.shape == 1 ? e.dims[2] : 0.0f};
      std::memcpy(&dims[3 * (size_t)i], dd, 12);
      sh[i] = e.shape; mat[i] = e.material_id; dyn[i] = e.body_type == 1; sok[i] = e.sleep_allowed != 0;
      im[i] = 0; in3[3 * i] = in3[3 * i + 1] = in3[3 * i + 2] = 0;
      if (dyn[i]) rp::mass_from_density(e.shape, dd, e.density, &im[i], &in3[3 * (size_t)i]);
    }
    uint32_t first = W->w->num_bodies();
    W->w->add_bodies_bulk(n, p7.data(), v6.data(), sh.data(), dims.data(), im.data(), in3.data(), dyn.data(), mat.data(),
                          sok.data());
    W->bodies_created += n;
    W->colliders_created += n;
    *out_first = first + 1;
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_add_bodies(RPhysWorld* W, const RPhysBodyDescEx* d, uint32_t n, uint32_t* out_first) {
  clear_err();
  if (out_first) *out_first = 0;
  if (!W || (!d && n) || !out_first) return fail(RPHYS_ERR_NULL, "rphys_ext_add_bodies: null arg");
  return add_bodies_impl(W, d, n, out_first, "rphys_ext_add_bodies", false, nullptr);
}
RPhysResult rphys_ext_batch_add_world(RPhysWorld* W, const RPhysBodyDescEx* d, uint32_t n, uint32_t* out_world,
                                      uint32_t* out_first) {
  clear_err();
  if (out_first) *out_first = 0;
  if (out_world) *out_world = 0;
  if (!W || !d || !out_first || !out_world) return fail(RPHYS_ERR_NULL, "rphys_ext_batch_add_world: null arg");
  return add_bodies_impl(W, d, n, out_first, "rphys_ext_batch_add_world", true, out_world);
}
RPhysResult rphys_ext_batch_num_worlds(const RPhysWorld* Wc, uint32_t* out) {
  clear_err();
  if (!Wc || !out) return fail(RPHYS_ERR_NULL, "rphys_ext_batch_num_worlds: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  LOCK;
  *out = W->w->batched() ? W->w->num_worlds() : 1u;
  return RPHYS_OK;
}
RPhysResult rphys_ext_batch_world_range(const RPhysWorld* Wc, uint32_t world, uint32_t* out_first, uint32_t* out_count) {
  clear_err();
  if (!Wc || !out_first || !out_count) return fail(RPHYS_ERR_NULL, "rphys_ext_batch_world_range: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  LOCK;
  *out_first = 0; *out_count = 0;
  uint32_t nw = W->w->batched() ? W->w->num_worlds() : 1u;
  if (world >= nw) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_batch_world_range: no such world");
  uint32_t b0 = W->w->batched() ? W->w->h_wb_start_[world] : 0u;
  uint32_t b1 = (W->w->batched() && world + 1 < nw) ? W->w->h_wb_start_[world + 1] : W->w->num_bodies();
  *out_first = b0 + 1;
  *out_count = b1 - b0;
  return RPHYS_OK;
}
RPhysResult rphys_ext_batch_get_hashes(const RPhysWorld* Wc, uint32_t first, uint32_t count, RPhysHash32* out) {
  clear_err();
  if (!Wc || (!out && count)) return fail(RPHYS_ERR_NULL, "rphys_ext_batch_get_hashes: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_ext_batch_get_hashes", [&]() {
    LOCK;
    uint32_t nw = W->w->batched() ? W->w->num_worlds() : 1u;
    if ((uint64_t)first + count > nw) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_batch_get_hashes: world range out of bounds");
    static_assert(sizeof(RPhysHash32) == 32, "RPhysHash32: 32 bytes");
    if (W->w->batched()) {
      // every requested world's digest from one pass of kernels over the world table
      W->w->step_hash_worlds(first, count, reinterpret_cast<uint8_t*>(out));
    } else {
      for (uint32_t k = 0; k < count; ++k) W->w->step_hash(out[k].bytes);
    }
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_set_pair_props(RPhysWorld* W, uint32_t a, uint32_t b, const RPhysPairProps* p) {
  clear_err();
  if (!W || !p) return fail(RPHYS_ERR_NULL, "rphys_ext_set_pair_props: null arg");
  if (!rp::material_known(a) || !rp::material_known(b)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_pair_props: unknown material");
  if (!(std::isfinite(p->mu_s) && std::isfinite(p->mu_k) && std::isfinite(p->restitution) && std::isfinite(p->stribeck_v)))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_pair_props: non-finite property");
  return guard("rphys_ext_set_pair_props", [&]() {
    LOCK;
    W->w->set_pair_props(a, b, rp::PairPropsHost{p->mu_s, p->mu_k, p->restitution, p->stribeck_v, 0.0f});
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_set_solver_iterations(RPhysWorld* W, uint32_t v, uint32_t p) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_solver_iterations: world is null");
  LOCK;
  W->w->set_solver_iterations(v, p);
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_gravity(RPhysWorld* W, RPhysVec3 g) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_gravity: world is null");
  LOCK;
  W->w->set_gravity(rp::mk3(g.x, g.y, g.z));
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_heightfield_f32(RPhysWorld* W, uint32_t nx, uint32_t nz, float cx, float cz, float ox, float oz,
                                          const float* h, uint32_t mat) {
  clear_err();
  if (!W || !h) return fail(RPHYS_ERR_NULL, "rphys_ext_set_heightfield_f32: null arg");
  if (nx == 0 || nz == 0) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_heightfield_f32: nx/nz == 0");
  if (!rp::material_known(mat)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_heightfield_f32: unknown material");
  std::vector<float> hh(h, h + (size_t)nx * nz);
  return guard("rphys_ext_set_heightfield_f32", [&]() {
    LOCK;
    return set_hf(W, nx, nz, cx, cz, ox, oz, std::move(hh), mat);
  });
}
// World::add_ball_joint / add_hinge_joint (world.rs:718-719) and D6 joints with every axis locked,
// all-or-nothing over the array.
RPhysResult rphys_ext_add_joints(RPhysWorld* W, const RPhysJointDesc* d, uint32_t n, uint32_t* out_first) {
  clear_err();
  if (out_first) *out_first = 0;
  if (!W || (!d && n) || !out_first) return fail(RPHYS_ERR_NULL, "rphys_ext_add_joints: null arg");
  LOCK;
  return guard("rphys_ext_add_joints", [&]() {
    std::vector<uint32_t> ab(2 * (size_t)n);
    for (uint32_t i = 0; i < n; ++i) {
      if (d[i].kind > RPHYS_JOINT_D6 || (d[i].kind == RPHYS_JOINT_HINGE && d[i].hinge_axis > 2))
        return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_joints: bad kind or hinge axis");
      if (!fin_iso(d[i].frame_a) || !fin_iso(d[i].frame_b))
        return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_joints: frame contains NaN/Inf");
      RPhysResult r = live_id(W, d[i].body_a, "rphys_ext_add_joints", &ab[2 * i]);
      if (r) return r;
      r = live_id(W, d[i].body_b, "rphys_ext_add_joints", &ab[2 * i + 1]);
      if (r) return r;
      if (ab[2 * i] == ab[2 * i + 1]) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_joints: body_a == body_b");
      if (W->w->batched() && W->w->num_worlds() > 0) {
        uint32_t wa = W->w->world_of(ab[2 * i]), wb = W->w->world_of(ab[2 * i + 1]);
        if (wa != wb) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_joints: in a batch, a joint joins two bodies of one world");
        uint32_t prev = i ? W->w->world_of(ab[2 * i - 2])
                          : (W->w->num_joints() ? W->w->world_of(W->w->h_joints_.back().a) : 0u);
        if (wa < prev) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_joints: in a batch, joints come in world order");
      }
    }
    *out_first = W->w->num_joints();
    for (uint32_t i = 0; i < n; ++i) {
      float fa[7], fb[7];
      pose7(d[i].frame_a, fa);
      pose7(d[i].frame_b, fb);
      W->w->add_joint(d[i].kind, ab[2 * i], ab[2 * i + 1], fa, fb, d[i].hinge_axis);
    }
    W->w->upload_joints();
    return RPHYS_OK;
  });
}
RPhysResult rphys_ext_add_distance_joints(RPhysWorld* W, const RPhysDistanceJointDesc* d, uint32_t n,
                                          uint32_t* out_first) {
  clear_err();
  if (out_first) *out_first = 0;
  if (!W || (!d && n) || !out_first) return fail(RPHYS_ERR_NULL, "rphys_ext_add_distance_joints: null arg");
  LOCK;
  return guard("rphys_ext_add_distance_joints", [&]() {
    std::vector<uint32_t> ab(2 * (size_t)n);
    auto fin3 = [](RPhysVec3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); };
    for (uint32_t i = 0; i < n; ++i) {
      if (!fin3(d[i].anchor_a) || !fin3(d[i].anchor_b) || !std::isfinite(d[i].rest) ||
          !(std::isfinite(d[i].compliance) && d[i].compliance >= 0.0f) ||
          !(std::isfinite(d[i].damping) && d[i].damping >= 0.0f))
        return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_distance_joints: non-finite value or negative compliance / damping");
      RPhysResult r = live_id(W, d[i].body_a, "rphys_ext_add_distance_joints", &ab[2 * i]);
      if (r) return r;
      r = live_id(W, d[i].body_b, "rphys_ext_add_distance_joints", &ab[2 * i + 1]);
      if (r) return r;
      if (ab[2 * i] == ab[2 * i + 1]) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_distance_joints: body_a == body_b");
      if (W->w->batched() && W->w->num_worlds() > 0) {
        uint32_t wa = W->w->world_of(ab[2 * i]), wb = W->w->world_of(ab[2 * i + 1]);
        if (wa != wb)
          return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_distance_joints: in a batch, a joint joins two bodies of one world");
        uint32_t prev = i ? W->w->world_of(ab[2 * i - 2])
                          : (W->w->num_joints() ? W->w->world_of(W->w->h_joints_.back().a) : 0u);
        if (wa < prev) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_add_distance_joints: in a batch, joints come in world order");
      }
    }
    *out_first = W->w->num_joints();
    for (uint32_t i = 0; i < n; ++i) {
      const float la[3] = {d[i].anchor_a.x, d[i].anchor_a.y, d[i].anchor_a.z};
      const float lb[3] = {d[i].anchor_b.x, d[i].anchor_b.y, d[i].anchor_b.z};
      W->w->add_distance_joint(ab[2 * i], ab[2 * i + 1], la, lb, d[i].rest, d[i].compliance, d[i].damping);
    }
    W->w->upload_joints();
    return RPHYS_OK;
  });
}
RPhysResult rphys_ext_set_joint_limit(RPhysWorld* W, uint32_t joint, uint32_t angular, uint32_t axis, uint32_t enabled,
                                      float lo, float hi) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_joint_limit: world is null");
  LOCK;
  if (joint >= W->w->num_joints()) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_set_joint_limit: joint out of range");
  if (axis > 2) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_limit: axis > 2");
  if (enabled && !(std::isfinite(lo) && std::isfinite(hi) && lo <= hi))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_limit: limit must be finite with lo <= hi");
  return guard("rphys_ext_set_joint_limit", [&]() {
    W->w->set_joint_limit(joint, angular != 0, axis, enabled != 0, lo, hi);
    W->w->upload_joints();
    return RPHYS_OK;
  });
}
RPhysResult rphys_ext_set_joint_limits(RPhysWorld* W, const RPhysJointLimit* l, uint32_t n) {
  clear_err();
  if (!W || (!l && n)) return fail(RPHYS_ERR_NULL, "rphys_ext_set_joint_limits: null arg");
  LOCK;
  for (uint32_t i = 0; i < n; ++i) {
    if (l[i].joint >= W->w->num_joints()) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_set_joint_limits: joint out of range");
    if (l[i].axis > 2) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_limits: axis > 2");
    if (l[i].enabled && !(std::isfinite(l[i].lo) && std::isfinite(l[i].hi) && l[i].lo <= l[i].hi))
      return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_limits: limit must be finite with lo <= hi");
  }
  return guard("rphys_ext_set_joint_limits", [&]() {
    for (uint32_t i = 0; i < n; ++i)
      W->w->set_joint_limit(l[i].joint, l[i].angular != 0, l[i].axis, l[i].enabled != 0, l[i].lo, l[i].hi);
    W->w->upload_joints();
    return RPHYS_OK;
  });
}
RPhysResult rphys_ext_set_joint_axis(RPhysWorld* W, uint32_t joint, uint32_t angular, uint32_t axis, uint32_t enabled,
                                     float compliance) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_joint_axis: world is null");
  LOCK;
  if (joint >= W->w->num_joints()) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_set_joint_axis: joint out of range");
  if (axis > 2) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_axis: axis > 2");
  if (!(std::isfinite(compliance) && compliance >= 0.0f))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_axis: compliance must be finite and >= 0");
  return guard("rphys_ext_set_joint_axis", [&]() {
    W->w->set_joint_axis(joint, angular != 0, axis, enabled != 0, compliance);
    W->w->upload_joints();
    return RPHYS_OK;
  });
}
RPhysResult rphys_ext_set_joint_drive(RPhysWorld* W, uint32_t joint, uint32_t angular, uint32_t axis,
                                      const RPhysJointDrive* d) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_joint_drive: world is null");
  LOCK;
  if (joint >= W->w->num_joints()) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_set_joint_drive: joint out of range");
  if (axis > 2) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_drive: axis > 2");
  if (d && !(std::isfinite(d->target) && std::isfinite(d->kp) && std::isfinite(d->kd) && std::isfinite(d->max_impulse)))
    return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_drive: non-finite drive value");
  return guard("rphys_ext_set_joint_drive", [&]() {
    if (d) W->w->set_joint_drive(joint, angular != 0, axis, true, d->target, d->kp, d->kd, d->max_impulse, d->vel_mode != 0);
    else W->w->set_joint_drive(joint, angular != 0, axis, false, 0.0f, 0.0f, 0.0f, 0.0f, false);
    W->w->upload_joints();
    return RPHYS_OK;
  });
}
RPhysResult rphys_ext_set_joint_damping(RPhysWorld* W, uint32_t joint, uint32_t angular, uint32_t axis, float damping,
                                        float friction) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_joint_damping: world is null");
  LOCK;
  if (joint >= W->w->num_joints()) return fail(RPHYS_ERR_INVALID_ID, "rphys_ext_set_joint_damping: joint out of range");
  if (axis > 2) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_joint_damping: axis > 2");
  return guard("rphys_ext_set_joint_damping", [&]() {
    W->w->set_joint_damping(joint, angular != 0, axis, damping, friction);
    W->w->upload_joints();
    return RPHYS_OK;
  });
}
RPhysResult rphys_ext_num_joints(const RPhysWorld* W, uint32_t* out) {
  clear_err();
  if (!W || !out) return fail(RPHYS_ERR_NULL, "rphys_ext_num_joints: null arg");
  *out = W->w->num_joints();
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_residual_mode(RPhysWorld* W, float tol, uint32_t max_sweeps) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_residual_mode: world is null");
  if (!std::isfinite(tol)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_residual_mode: tolerance not finite");
  LOCK;
  W->w->set_residual_mode(tol, max_sweeps);
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_solve_order(RPhysWorld* W, uint32_t order) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_solve_order: world is null");
  if (order > RPHYS_ORDER_COLOURED) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_solve_order: unknown order");
  LOCK;
  W->w->set_coloured(order == RPHYS_ORDER_COLOURED);
  return RPHYS_OK;
}
static bool tuning_ok(const RPhysTuning& t) {
  auto in = [](uint32_t v, uint32_t a, uint32_t b, uint32_t c) { return v == a || v == b || v == c; };
  return (in(t.group_rows, 8, 16, 32) || in(t.group_rows, 64, 128, 128)) && in(t.packed_threads, 32, 64, 128) &&
         (t.island_threads == 32 || in(t.island_threads, 64, 128, 256));
}
RPhysResult rphys_ext_set_tuning(RPhysWorld* W, const RPhysTuning* t) {
  clear_err();
  if (!W || !t) return fail(RPHYS_ERR_NULL, "rphys_ext_set_tuning: null arg");
  if (!tuning_ok(*t)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_set_tuning: unsupported launch shape");
  LOCK;
  W->w->tuning_.group_rows = t->group_rows;
  W->w->tuning_.packed_threads = t->packed_threads;
  W->w->tuning_.island_threads = t->island_threads;
  return RPHYS_OK;
}
RPhysResult rphys_ext_get_tuning(const RPhysWorld* Wc, RPhysTuning* out) {
  clear_err();
  if (!Wc || !out) return fail(RPHYS_ERR_NULL, "rphys_ext_get_tuning: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  LOCK;
  *out = RPhysTuning{W->w->tuning_.group_rows, W->w->tuning_.packed_threads, W->w->tuning_.island_threads};
  return RPHYS_OK;
}
RPhysResult rphys_ext_step_n(RPhysWorld* W, float dt, uint32_t n) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_step_n: world is null");
  if (!std::isfinite(dt) || dt < 0) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_step_n: bad dt");
  return guard("rphys_ext_step_n", [&]() {
    LOCK;
    for (uint32_t i = 0; i < n; ++i) W->w->step(dt);
    W->w->synchronize();
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_get_stats(const RPhysWorld* Wc, RPhysStepStats* o) {
  clear_err();
  if (!Wc || !o) return fail(RPHYS_ERR_NULL, "rphys_ext_get_stats: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_ext_get_stats", [&]() {
    LOCK;
    const rp::StepStatsHost& s = W->w->stats();
    o->pairs = s.pairs; o->contacts = s.contacts; o->islands = s.islands; o->levels = s.levels;
    o->max_batch = s.max_batch; o->warm_matched = s.warm_matched; o->sweeps = s.sweeps;
    o->bounce_rows = s.bounce_rows; o->warm_entries = s.warm_entries; o->sleeping = s.sleeping;
    o->error_flags = s.error_flags; o->residual = s.residual;
    o->row_sweeps = s.row_sweeps; o->rows_scheduled = s.rows_scheduled;
    o->groups_shared = s.groups_shared; o->groups_global = s.groups_global;
    o->max_group_rows = s.max_group_rows; o->max_group_bodies = s.max_group_bodies;
    o->islands_capped = s.islands_capped;
    o->pred_used = s.pred_used;
    o->rows_capped = s.rows_capped;
    for (int k = 0; k < 6; ++k) o->res_hist[k] = s.res_hist[k];
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_get_pairs(const RPhysWorld* Wc, uint32_t* out, uint32_t cap, uint32_t* out_count) {
  clear_err();
  if (!Wc || !out_count) return fail(RPHYS_ERR_NULL, "rphys_ext_get_pairs: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_ext_get_pairs", [&]() {
    LOCK;
    std::vector<uint64_t> p;
    W->w->get_pairs(p);
    *out_count = (uint32_t)p.size();
    if (!out) return (RPhysResult)RPHYS_OK;
    for (uint32_t i = 0; i < p.size() && i < cap; ++i) { out[2 * i] = (uint32_t)(p[i] >> 32); out[2 * i + 1] = (uint32_t)p[i]; }
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_get_contact_records(const RPhysWorld* Wc, RPhysContactRecord* out, uint32_t cap, uint32_t* out_count) {
  clear_err();
  if (!Wc || !out_count) return fail(RPHYS_ERR_NULL, "rphys_ext_get_contact_records: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_ext_get_contact_records", [&]() {
    LOCK;
    std::vector<WorldGpu::ContactOut> cs;
    W->w->get_contacts(cs);
    *out_count = (uint32_t)cs.size();
    if (!out) return (RPhysResult)RPHYS_OK;
    for (uint32_t i = 0; i < cs.size() && i < cap; ++i) {
      const auto& c = cs[i];
      RPhysContactRecord r;
      r.a_collider = c.a; r.b_collider = c.b;
      r.point = RPhysVec3{c.p[0], c.p[1], c.p[2]};
      r.normal = RPhysVec3{c.n[0], c.n[1], c.n[2]};
      r.depth = c.depth; r.impulse = c.impulse; r.level = c.level; r.pad = 0;
      out[i] = r;
    }
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_get_body_states(const RPhysWorld* Wc, uint32_t first, uint32_t count, float* out) {
  clear_err();
  if (!Wc || (!out && count)) return fail(RPHYS_ERR_NULL, "rphys_ext_get_body_states: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_ext_get_body_states", [&]() {
    LOCK;
    if ((uint64_t)first + count > W->w->num_bodies()) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_get_body_states: range out of bounds");
    W->w->get_body_states(first, count, out);
    return (RPhysResult)RPHYS_OK;
  });
}

RPhysResult rphys_ext_profile_enable(RPhysWorld* W, uint32_t on) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_profile_enable: world is null");
  LOCK;
  W->w->profile_enable(on != 0);
  return RPHYS_OK;
}
RPhysResult rphys_ext_profile_read(const RPhysWorld* Wc, double* ms, uint64_t* ticks, uint32_t cap, uint32_t* out_n) {
  clear_err();
  if (!Wc || !out_n) return fail(RPHYS_ERR_NULL, "rphys_ext_profile_read: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  LOCK;
  std::vector<double> m(64);
  std::vector<uint64_t> c(64);
  int n = W->w->profile_read(m.data(), c.data(), 64);
  *out_n = (uint32_t)n;
  for (int i = 0; i < n && (uint32_t)i < cap; ++i) {
    if (ms) ms[i] = m[i];
    if (ticks) ticks[i] = c[i];
  }
  return RPHYS_OK;
}
const char* rphys_ext_profile_stage_name(uint32_t stage) { return WorldGpu::phase_name((int)stage); }

RPhysResult rphys_ext_stream_handle(const RPhysWorld* Wc, uint64_t* out) {
  clear_err();
  if (!Wc || !out) return fail(RPHYS_ERR_NULL, "rphys_ext_stream_handle: null arg");
  *out = (uint64_t)(uintptr_t)Wc->w->stream();
  return RPHYS_OK;
}

RPhysResult rphys_ext_launch_count(uint64_t* out) {
  clear_err();
  if (!out) return fail(RPHYS_ERR_NULL, "rphys_ext_launch_count: null arg");
  *out = rp::g_launches;
  return RPHYS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- learned warm-start model
struct RPhysWarmModel {
  std::mutex mu;
  std::unique_ptr<rp::WarmModel> m;
  std::mutex& m_mu() { return mu; }
};
extern "C" {
RPhysWarmModel* rphys_ext_model_create(uint64_t seed) {
  clear_err();
  try {
    auto* M = new RPhysWarmModel();
    M->m.reset(new rp::WarmModel(seed));
    return M;
  } catch (const std::exception& e) {
    fail(RPHYS_ERR_INTERNAL, std::string("rphys_ext_model_create: ") + e.what());
    return nullptr;
  }
}
void rphys_ext_model_destroy(RPhysWarmModel* M) {
  try { delete M; } catch (...) {}
}
uint32_t rphys_ext_model_num_params(void) { return rp::WarmModel::kParams; }
RPhysResult rphys_ext_model_get_weights(const RPhysWarmModel* Mc, float* out, uint32_t n) {
  clear_err();
  if (!Mc || !out) return fail(RPHYS_ERR_NULL, "rphys_ext_model_get_weights: null arg");
  if (n != rp::WarmModel::kParams) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_model_get_weights: count != num_params");
  auto* M = const_cast<RPhysWarmModel*>(Mc);
  return guard("rphys_ext_model_get_weights", [&]() { std::lock_guard<std::mutex> g(M->mu); M->m->get_weights(out); return (RPhysResult)RPHYS_OK; });
}
RPhysResult rphys_ext_model_set_weights(RPhysWarmModel* M, const float* in, uint32_t n) {
  clear_err();
  if (!M || !in) return fail(RPHYS_ERR_NULL, "rphys_ext_model_set_weights: null arg");
  if (n != rp::WarmModel::kParams) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_model_set_weights: count != num_params");
  for (uint32_t i = 0; i < n; ++i)
    if (!std::isfinite(in[i])) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_model_set_weights: non-finite weight");
  return guard("rphys_ext_model_set_weights", [&]() { std::lock_guard<std::mutex> g(M->mu); M->m->set_weights(in); return (RPhysResult)RPHYS_OK; });
}
RPhysResult rphys_ext_model_predict(RPhysWarmModel* M, const float* f, uint32_t n, float* out) {
  clear_err();
  if (!M || (n && (!f || !out))) return fail(RPHYS_ERR_NULL, "rphys_ext_model_predict: null arg");
  return guard("rphys_ext_model_predict", [&]() { std::lock_guard<std::mutex> g(M->mu); M->m->predict(n, f, out, false); return (RPhysResult)RPHYS_OK; });
}
RPhysResult rphys_ext_model_predict_device(RPhysWarmModel* M, const float* d_f, uint32_t n, float* d_out, uint64_t stream) {
  clear_err();
  if (!M || (n && (!d_f || !d_out))) return fail(RPHYS_ERR_NULL, "rphys_ext_model_predict_device: null arg");
  return guard("rphys_ext_model_predict_device", [&]() {
    std::lock_guard<std::mutex> g(M->m_mu());
    M->m->predict(n, d_f, d_out, true, reinterpret_cast<cudaStream_t>(stream));
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_model_gradients(RPhysWarmModel* M, const float* f, const float* t, uint32_t n, float* grads, float* loss) {
  clear_err();
  if (!M || !f || !t || !grads || !loss || !n) return fail(RPHYS_ERR_NULL, "rphys_ext_model_gradients: null arg or no rows");
  return guard("rphys_ext_model_gradients", [&]() {
    std::lock_guard<std::mutex> g(M->mu);
    *loss = M->m->gradients(n, f, t, false);
    M->m->get_grads(grads);
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_model_train(RPhysWarmModel* M, const float* f, const float* t, uint32_t n, uint32_t epochs, uint32_t batch,
                                  float lr, float* loss) {
  clear_err();
  if (!M || !f || !t || !loss || !n) return fail(RPHYS_ERR_NULL, "rphys_ext_model_train: null arg or no rows");
  if (batch == 0 || !(std::isfinite(lr) && lr > 0)) return fail(RPHYS_ERR_BAD_ARG, "rphys_ext_model_train: batch > 0 and lr > 0");
  return guard("rphys_ext_model_train", [&]() {
    std::lock_guard<std::mutex> g(M->mu);
    *loss = M->m->train(n, f, t, epochs, batch, lr);
    return (RPhysResult)RPHYS_OK;
  });
}
}  // extern "C"

// ---------------------------------------------------------------- learned warm start in a world
extern "C" {
RPhysResult rphys_ext_set_warm_model(RPhysWorld* W, RPhysWarmModel* M) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_warm_model: world is null");
  LOCK;
  W->w->model_ = M ? M->m.get() : nullptr;
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_warm_policy(RPhysWorld* W, uint32_t cold_only) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_warm_policy: world is null");
  LOCK;
  W->w->pred_cold_only_ = cold_only != 0;
  return RPHYS_OK;
}
RPhysResult rphys_ext_set_feature_logging(RPhysWorld* W, uint32_t on) {
  clear_err();
  if (!W) return fail(RPHYS_ERR_NULL, "rphys_ext_set_feature_logging: world is null");
  LOCK;
  W->w->feat_log_ = on != 0;
  return RPHYS_OK;
}
RPhysResult rphys_ext_get_row_features(const RPhysWorld* Wc, float* feats, float* targets, uint32_t cap, uint32_t* out_n) {
  clear_err();
  if (!Wc || !out_n) return fail(RPHYS_ERR_NULL, "rphys_ext_get_row_features: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_ext_get_row_features", [&]() {
    LOCK;
    std::vector<float> f, t;
    W->w->get_row_features(f, t);
    uint32_t n = (uint32_t)(t.size() / 3);
    *out_n = n;
    if (feats && targets)
      for (uint32_t i = 0; i < n && i < cap; ++i) {
        std::memcpy(feats + 24 * (size_t)i, f.data() + 24 * (size_t)i, 96);
        std::memcpy(targets + 3 * (size_t)i, t.data() + 3 * (size_t)i, 12);
      }
    return (RPhysResult)RPHYS_OK;
  });
}
RPhysResult rphys_ext_get_row_predictions(const RPhysWorld* Wc, float* out4, uint32_t cap, uint32_t* out_n) {
  clear_err();
  if (!Wc || !out_n) return fail(RPHYS_ERR_NULL, "rphys_ext_get_row_predictions: null arg");
  RPhysWorld* W = const_cast<RPhysWorld*>(Wc);
  return guard("rphys_ext_get_row_predictions", [&]() {
    LOCK;
    std::vector<float> p;
    W->w->get_row_predictions(p);
    uint32_t n = (uint32_t)(p.size() / 4);
    *out_n = n;
    if (out4) std::memcpy(out4, p.data(), 16 * (size_t)(n < cap ? n : cap));
    return (RPhysResult)RPHYS_OK;
  });
}
}  // extern "C"
