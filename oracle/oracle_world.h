// oracle/oracle_world.h -- TEST INFRASTRUCTURE (the oracle): a CPU restatement of the
// reference's per-tick rigid-body step, World::step (riftphys-world/src/world/step.rs:40-542)
// and everything it calls at the configured feature set: sphere / box / capsule colliders with
// no offset, a static ground body, a HeightField environment, rigid contacts, warm starting,
// sleeping, the BLAKE3 tick hash. Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg use it; the product (riftphys-rust_b200/) never links it.
//
// Joints: D6 joints (ball, hinge, per-axis limits; riftphys-articulation/src/bodies.rs:326-391)
// with their velocity rows (solver.rs:291-424, 644-687, 699-712, 788-834, 946-952) and the XPBD
// position pass with SHAKE directions (bodies.rs:422-471, 616-873). Drives, compliance, joint
// damping / friction, armature and distance joints are not restated.
// Not restated (no configuration reaches them, or the C ABI cannot): compliant and
// patch-friction pairs, collider offsets, players, accel components, pending epoch swaps. The
// W6 bounce passes (solver.rs:1047-1241) are detected and counted, and the rows that would take
// them are left as the inelastic solve produced them (the same rule the GPU path follows).
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "om.h"

namespace orc {
using om::M3;
using om::Q4;
using om::V3;

enum : uint32_t { SH_SPHERE = 0, SH_BOX = 1, SH_CAPSULE = 2, SH_TRIANGLE = 3 };
static const uint32_t kTerrain = 0xFFFFFFFFu;  // TERRAIN_CI (world.rs:26)

struct Shape { uint32_t kind; float a, b, c; V3 ta, tb, tc; };
struct Aabb { V3 min, max; };
struct Iso { V3 pos; Q4 rot; };
struct Collider { uint32_t body; Shape shape; Aabb aabb; uint32_t mat; };
struct Contact {
  uint32_t a_collider, b_collider;
  V3 point, normal;
  float depth;
  int32_t env_mat;  // -1: None
  float impulse;
};
struct PairProps { float mu_s, mu_k, restitution, stribeck_v, stiffness; };
using WarmKey = std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>;
struct WarmContact { V3 la; float jn; V3 jt; };

struct HeightField {
  uint32_t nx = 0, nz = 0;
  float sx = 1, sz = 1, ox = 0, oz = 0;
  std::vector<float> h;
  float min_y = 0, max_y = 0;
  uint32_t mat = 4;
};

// D6 joint (bodies.rs:55-137) at the restated feature set: an axis is enabled or free, with an
// optional limit [lo, hi], XPBD compliance, an optional drive (position target, or a velocity motor
// with its impulse cap), viscous damping and Coulomb friction; hinge is the stored hinge axis
// (add_hinge) or -1. Armature is not restated.
struct D6Axis {
  bool enabled = false, has_limit = false;
  float lo = 0.0f, hi = 0.0f;
  float compliance = 0.0f, damping = 0.0f, friction = 0.0f;
  bool has_drive = false, vel_mode = false;
  float d_target = 0.0f, d_kp = 0.0f, d_kd = 0.0f, d_max = 0.0f;
};
// JointKind (bodies.rs:140-143): a D6 joint (kind 0) or a distance joint (kind 1,
// DistanceJoint, bodies.rs:31-51: rest length, compliance, anchors la / lb in each body's frame,
// damping along the rod; both anchors zero and no damping is the original COM-to-COM joint).
struct Joint {
  uint32_t a, b;
  int kind = 0;
  Iso fa, fb;
  D6Axis t[3], r[3];
  int hinge = -1;
  float lam_t[3] = {0, 0, 0}, lam_r[3] = {0, 0, 0};  // XPBD multipliers of the current step
  float rest = 0.0f, compliance = 0.0f, damping = 0.0f, lambda_acc = 0.0f;
  V3 la{0, 0, 0}, lb{0, 0, 0};
  // DistanceJoint::anchored (bodies.rs:47-51)
  bool anchored() const {
    return !(la.x == 0.0f && la.y == 0.0f && la.z == 0.0f) || !(lb.x == 0.0f && lb.y == 0.0f && lb.z == 0.0f) ||
           damping > 0.0f;
  }
};
// warm_joints entry (solver.rs:946-952): per row, its tag and accumulated impulse
using WarmJointRows = std::vector<std::pair<uint8_t, float>>;

struct CarriedState {
  std::map<WarmKey, std::vector<WarmContact>> warm;
  std::map<uint32_t, WarmJointRows> warm_joints;
  std::vector<V3> last_lin_vel;
  std::vector<uint8_t> awake;
  std::vector<uint16_t> sleep_ticks;
};

struct Snapshot {
  uint64_t tick;
  std::vector<Iso> poses;
  std::vector<V3> lin, ang;
  CarriedState carried;
};

struct Stats {
  uint32_t pairs = 0, contacts = 0, islands = 0, levels = 0, max_batch = 0, warm_matched = 0;
  uint32_t sweeps = 0, bounce_rows = 0, row_sweeps = 0, rows_scheduled = 0;
  uint32_t islands_capped = 0;  // residual mode: solve islands still above the tolerance at the cap
  uint32_t pred_used = 0;       // rows started from an offered prediction
  uint32_t rows_capped = 0;     // residual mode: rows of the islands counted in islands_capped
  uint32_t res_hist[6] = {0, 0, 0, 0, 0, 0};  // solve islands by last-sweep residual (res_bin)
  float residual = 0;
};

// Unit of the learned warm start's impulses (a row's effective mass x 9.81 / 60), one f32 constant.
constexpr float kImpulseUnit = 0.1635f;

struct World {
  V3 gravity{0.0f, -9.81f, 0.0f};
  uint64_t epoch = 0;
  uint64_t rng = 0xC0FFEEull | 1ull;
  // Bodies SoA (riftphys-dynamics/src/dynamics.rs:38-46)
  std::vector<V3> pos;
  std::vector<Q4> rot;
  std::vector<V3> lin, ang;
  std::vector<float> inv_mass;
  std::vector<uint8_t> dyn;
  std::vector<M3> inv_I;
  std::vector<Collider> colliders;
  // SleepManager (sleep.rs:5-13): sized to the world's capacity at creation
  std::vector<uint8_t> awake, sleep_allowed;
  std::vector<uint16_t> sleep_ticks;
  std::vector<uint8_t> alive;
  std::vector<V3> last_lin_vel;
  std::map<WarmKey, std::vector<WarmContact>> warm;
  std::vector<Joint> joints;
  std::map<uint32_t, WarmJointRows> warm_joints;
  uint32_t iters_v = 20, iters_p = 20;
  std::vector<std::pair<std::pair<uint32_t, uint32_t>, PairProps>> overrides;
  bool has_hf = false;
  HeightField hf;
  uint64_t tick = 0;
  std::vector<Contact> last_frame_contacts;
  std::vector<std::pair<uint32_t, uint32_t>> last_pairs;
  std::vector<uint32_t> last_levels;  // per last_frame_contacts entry
  Stats stats;
  float res_tol = 0.0f;
  // Solve order (an extension): false, the reference's serial order (its level schedule); true,
  // coloured order for worlds without joints (see the tick's colouring step).
  bool coloured = false;
  // predictions offered to the next tick's warm start, 4 floats per contact in contact order
  // (normal, friction 1, friction 2 in kImpulseUnit x m_n; 1 when offered), consumed by step()
  std::vector<float> next_pred;
  uint32_t res_max = 0;
  int threads = 1;  // >1: narrowphase and level batches on OpenMP (order-preserving)
  // Diagnostics of the residual stop (test infrastructure only): when on, the velocity solve keeps,
  // for the island with the largest last-sweep residual, its rows (bodies, m_n, jn, residual)
  // and its residual after every sweep.
  bool diag_worst = false;
  std::vector<float> diag_rows;   // 5 per row: body a, body b (as float bits), m_n, jn, last residual
  std::vector<float> diag_hist;   // residual per sweep

  explicit World(uint32_t capacity);
  uint32_t num_bodies() const { return (uint32_t)pos.size(); }

  // dynamics.rs
  M3 inv_inertia_world(uint32_t i) const;
  void set_pose(uint32_t i, const Iso& p);
  void set_vel(uint32_t i, V3 l, V3 a);
  void apply_impulse(uint32_t i, V3 j);
  void apply_angular_impulse(uint32_t i, V3 tau);
  // world.rs
  uint32_t add_body(const Iso& pose, V3 lin, V3 ang, float inv_mass_in, V3 inertia_diag,
                    bool dynamic);
  void add_collider(uint32_t body, const Shape& s, uint32_t mat);
  void set_body_pose(uint32_t id, const Iso& p);
  void set_body_vel(uint32_t id, V3 l, V3 a);
  void wake(uint32_t id);
  void apply_impulse_world(uint32_t id, V3 j);
  bool remove_body(uint32_t id);
  void drop_warm_of(uint32_t b);
  // joints (world.rs:718-720, 966-968; bodies.rs:326-391)
  uint32_t add_ball_joint(uint32_t a, uint32_t b, const Iso& fa, const Iso& fb);
  uint32_t add_hinge_joint(uint32_t a, uint32_t b, const Iso& fa, const Iso& fb, uint32_t axis);
  void set_d6_limit(uint32_t id, bool angular, uint32_t axis, bool has, float lo, float hi);
  // World::add_d6_joint (world.rs:720-725) with every axis enabled (locked) and no stored hinge axis
  uint32_t add_d6_joint(uint32_t a, uint32_t b, const Iso& fa, const Iso& fb);
  // D6Axis.enabled / .compliance as add_d6_joint's struct sets them
  void set_d6_axis(uint32_t id, bool angular, uint32_t axis, bool enabled, float compliance);
  // set_d6_drive_t / set_d6_drive_r (bodies.rs:354-366) and set_d6_damping (:376-383)
  void set_d6_drive(uint32_t id, bool angular, uint32_t axis, bool has, float target, float kp, float kd,
                    float max_impulse, bool vel_mode);
  void set_d6_damping(uint32_t id, bool angular, uint32_t axis, float damping, float friction);
  // Joints::add_distance_joint / add_distance_joint_at / set_distance_damping (bodies.rs:273-305)
  uint32_t add_distance_joint(uint32_t a, uint32_t b, float rest, float compliance);
  uint32_t add_distance_joint_at(uint32_t a, V3 la, uint32_t b, V3 lb, float rest, float compliance);
  void set_distance_damping(uint32_t id, float damping);
  PairProps pair_props(uint32_t a, uint32_t b) const;
  void set_pair_props(uint32_t a, uint32_t b, const PairProps& p);
  void update_colliders_aabb();
  CarriedState carried_state() const;
  void restore_carried_state(const CarriedState& s);
  // PlayerController (world.rs:45-70) and World::add_player (world.rs:466-475): a static body with a
  // capsule collider of the controller's default size (radius 0.4, half height 0.9), whatever size
  // the controller is given afterwards.
  struct Player { uint32_t body; float radius = 0.4f, height = 1.8f, speed = 5.0f; bool grounded = false;
                  float vertical_vel = 0.0f; V3 input{0, 0, 0}; };
  std::vector<Player> players;
  uint32_t add_player(const Iso& pose);
  void update_players(float dt);  // step.rs:544-639
  // World::raycast (queries.rs:50-116): dir normalised here again; ignore a body index or
  // 0xFFFFFFFF. Returns false on a miss; body 0xFFFFFFFF is the terrain.
  bool raycast(V3 origin, V3 dir, float max_dist, uint32_t ignore, uint32_t* body, float* toi, V3* point,
               V3* normal) const;
  // World::raycast_exact (queries.rs:18-48) with the skip set to one body index (0xFFFFFFFF: none)
  bool raycast_exact(V3 origin, V3 dir, float max_dist, uint32_t ignore, uint32_t* body, float* toi, V3* point,
                     V3* normal) const;
  // World::sweep_capsule (queries.rs:118-249): a y-axis capsule from -> to. Returns false on a
  // miss; body 0xFFFFFFFF is the terrain; *overlap when it started overlapping (toi 0).
  bool sweep_capsule(V3 from, V3 to, float radius, float half_height, uint32_t ignore, uint32_t* body, float* toi,
                     bool* overlap, V3* point, V3* normal) const;
  // step.rs / provenance.rs
  void step(float dt);
  void step_hash(uint8_t out[32]) const;
  uint32_t num_sleeping() const;
};

Aabb aabb_of(const Shape& s, const Iso& xf);

// Narrowphase (riftphys-collision/src/narrowphase.rs), exposed for unit tests.
struct CP { V3 position, normal; float penetration; };
struct Manifold { V3 normal; CP pts[4]; int len = 0; };
bool collide_shapes(const Shape& a, const Iso& xa, const Shape& b, const Iso& xb, float cd, Manifold* out);

// MassProps::from_*_density (riftphys-geom/src/mass.rs:75-145): inv_mass and inertia diagonal.
bool mass_from_density(uint32_t shape, const float dims[3], float density, float* inv_mass, V3* inertia);
// Material table and pair mixing (riftphys-materials/src/materials.rs:97-101,278-305)
PairProps table_pair_props(uint32_t a, uint32_t b);
bool material_known(uint32_t id);

}  // namespace orc
