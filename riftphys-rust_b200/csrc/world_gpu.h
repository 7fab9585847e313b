// world_gpu.h -- the device-resident world behind the C ABI, and the per-tick pipeline that
// replaces World::step (riftphys-world/src/world/step.rs:40-420) on one B200.
//
// HBM layout (structure of arrays, 16-byte rows for 128-bit loads):
//   bodies     pos/rot/lin/ang/last_lin float4, inv_mass f32, inv_I 9 x f32 (column-major),
//              dyn/awake/sleep_allowed/alive u8, sleep_ticks u16 -- allocated at the world's
//              body capacity; sleep arrays are hashed at that length, as the reference sizes
//              SleepManager by capacity (sleep.rs:15-27).
//   colliders  body u32, kind u32, mat u32, dims float4 (one collider per body, body order).
//   warm cache sorted by key (uint4: body A, body B or 0xFFFFFFFF, ordinal A, ordinal B);
//              la+jn float4, jt float4 per entry, entries of one key contiguous in contact order.
//   per tick   pairs (u64 (i << 32 | j)), contacts (SoA), rows (SoA), schedules (u32 arrays).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "rp_math.cuh"

namespace rp {

class WarmModel;
struct JointGpu;
// Most velocity rows one D6 joint has: 6 axes x (damper, friction, motor, two limit rows), rounded up.
constexpr uint32_t kJointRows = 32;

struct StepStatsHost {
  uint32_t pairs = 0, contacts = 0, islands = 0, levels = 0, max_batch = 0, warm_matched = 0;
  uint32_t sweeps = 0, bounce_rows = 0, warm_entries = 0, sleeping = 0, error_flags = 0;
  float residual = 0.0f;
  uint32_t row_sweeps = 0, rows_scheduled = 0;
  uint32_t groups_shared = 0, groups_global = 0, max_group_rows = 0, max_group_bodies = 0;
  uint32_t islands_capped = 0, pred_used = 0;
  uint32_t rows_capped = 0, res_hist[6] = {0, 0, 0, 0, 0, 0};
};

struct PairPropsHost { float mu_s, mu_k, restitution, stribeck_v, stiffness; };

// A device array that only grows.
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t cap = 0;
  void ensure(size_t n);
  void release();
  ~DBuf() { release(); }
};

// PlayerController (world.rs:45-70) as the device keeps it, 16 words: the controller's state, its
// input, and the pose its body had when the tick's player pass began.
struct PlayerGpu {
  uint32_t body;
  float radius, height, speed;
  float vvel;
  uint32_t grounded;
  float in[3];
  float p0[3], q0[4];
};
static_assert(sizeof(PlayerGpu) == 64, "PlayerGpu: 16 words");

struct SnapshotGpu;

class WorldGpu {
 public:
  WorldGpu(uint32_t max_bodies, uint32_t max_colliders);
  ~WorldGpu();

  // ---- configuration and body management (world.rs)
  uint32_t num_bodies() const { return nb_; }
  uint32_t num_colliders() const { return ncol_; }
  uint32_t capacity() const { return cap_b_; }
  bool alive(uint32_t id) const { return id < nb_ && h_alive_[id] != 0; }
  // World::add_body + add_collider; shape/dims/material as RPhysBodyDescEx. Returns the index.
  uint32_t add_body(const float pose[7], const float vel[6], uint32_t shape, const float dims[3],
                    float inv_mass, const float inertia_diag[3], bool dynamic, uint32_t mat,
                    bool sleep_allowed);
  void add_bodies_bulk(uint32_t n, const float* pose7, const float* vel6, const uint32_t* shape,
                       const float* dims3, const float* inv_mass, const float* inertia3,
                       const uint8_t* dynamic, const uint32_t* mat, const uint8_t* sleep_allowed);
  bool remove_body(uint32_t id);
  void set_body_pose(uint32_t id, const float pose[7]);
  void set_body_vel(uint32_t id, const float vel[6]);
  void apply_impulse(uint32_t id, const float j[3]);
  void get_body_pose(uint32_t id, float pose[7]);
  void get_body_vel(uint32_t id, float vel[6]);
  void get_body_states(uint32_t first, uint32_t count, float* out13);
  void set_pair_props(uint32_t a, uint32_t b, const PairPropsHost& p);
  void set_solver_iterations(uint32_t v, uint32_t p) { iters_v_ = v < 1 ? 1 : v; iters_p_ = p < 1 ? 1 : p; }
  void set_gravity(f3 g) { gravity_ = g; }
  void set_residual_mode(float tol, uint32_t max_sweeps) { res_tol_ = tol; res_max_ = max_sweeps; }
  // Solve order: false, the reference's serial order (exact); true, coloured (worlds without joints)
  void set_coloured(bool on) { coloured_ = on; }
  bool coloured_ = false;
  // Launch shapes of the velocity solve (none changes a result bit: islands are independent and the
  // rows of a level are): rows up to which islands are packed into shared groups (8, 16, 32), threads
  // of a packed-group block (32, 64, 128) and of a single-island block (32, 64, 128, 256). Defaults are
  // the autotuner's choice for the terrain workload.
  struct Tuning { uint32_t group_rows = 64, packed_threads = 32, island_threads = 128; };
  Tuning tuning_;
  void set_heightfield(uint32_t nx, uint32_t nz, float sx, float sz, float ox, float oz,
                       const std::vector<float>& q6_heights, float min_y, float max_y, uint32_t mat);
  void clear_heightfield();
  void set_epoch(uint64_t e) { epoch_ = e; }
  void set_rng_state(uint64_t s) { rng_ = s; }
  uint64_t tick() const { return tick_; }

  // ---- the tick
  void step(float dt);      // World::step, asynchronous on the world's stream
  void synchronize();       // waits for the stream; raises on a device error
  void step_hash(uint8_t out[32]);
  // The same digest with every scratch byte in one fixed device array (hash.cu); allocates
  // nothing. Throws std::length_error when the world does not fit that array.
  void step_hash_noalloc(uint8_t out[32]);

  // ---- batched worlds: independent worlds in contiguous body / collider ranges of one device
  // world. Bodies of different worlds never pair in the broadphase; every later stage works per
  // island already, so nothing else couples them.
  void begin_world();                                   // bodies added next form a new world
  uint32_t num_worlds() const { return (uint32_t)h_wb_start_.size(); }
  bool batched() const { return batch_; }
  void step_hash_world(uint32_t w, uint8_t out[32]);    // that world's own digest
  // the digests of worlds [first, first + count), 32 bytes each, from kernels over the world table
  void step_hash_worlds(uint32_t first, uint32_t count, uint8_t* out);
  std::vector<uint32_t> h_wb_start_, h_wc_start_;       // first body / collider of each world
  bool batch_ = false, worlds_dirty_ = false;
  DBuf<uint32_t> col_world, world_col_start;           // per collider; per world (+ end)
  void upload_worlds();

  // ---- D6 joints (world.rs:718-720, 966-968; bodies.rs:326-391): ball and hinge joints with
  // per-axis limits. Joint ids are 0-based in creation order. In a batch, a joint joins two
  // bodies of one world and joints come in world order, so each world's joints form one
  // contiguous id range.
  struct JointHost {
    uint32_t a, b;
    float fa[7], fb[7];            // frame in body A / B: pos xyz, quat xyzw
    bool en[6], lim[6];            // t0 t1 t2 r0 r1 r2
    float lo[6], hi[6];
    float comp[6], damp[6], fric[6];  // XPBD compliance, damping, Coulomb friction
    bool drive[6], vel[6];         // driven; the drive a velocity motor
    float dtarget[6], dkp[6], dkd[6], dmax[6];
    int hinge;                     // stored hinge axis (add_hinge), -1 none
    // kind 1, a distance joint: rest length, compliance, damping along the rod; anchors in fa / fb
    int kind;
    float rest, dcomp, ddamp;
  };
  uint32_t num_joints() const { return (uint32_t)h_joints_.size(); }
  uint32_t world_of(uint32_t body) const;
  uint32_t add_joint(uint32_t kind, uint32_t a, uint32_t b, const float fa[7], const float fb[7], uint32_t axis);
  void set_joint_limit(uint32_t j, bool angular, uint32_t axis, bool on, float lo, float hi);
  void set_joint_axis(uint32_t j, bool angular, uint32_t axis, bool enabled, float compliance);
  void set_joint_drive(uint32_t j, bool angular, uint32_t axis, bool on, float target, float kp, float kd,
                       float max_impulse, bool vel_mode);
  void set_joint_damping(uint32_t j, bool angular, uint32_t axis, float damping, float friction);
  uint32_t add_distance_joint(uint32_t a, uint32_t b, const float la[3], const float lb[3], float rest, float compliance,
                              float damping);
  void upload_joints();            // the joint records, jointed bodies and jointed pairs, on change
  std::vector<JointHost> h_joints_;
  bool joints_dirty_ = false;
  uint32_t jw_init_ = 0;                       // joints whose cache entry is initialised
  DBuf<JointGpu> joints_d;
  DBuf<uint8_t> jointed_d;                     // per body: in some joint
  DBuf<unsigned long long> jpair_keys;         // (min body << 32 | max body), sorted, unique
  uint32_t n_jpairs = 0;
  // the joint warm cache (warm_joints, solver.rs:946-952): per joint the row count (0xFFFFFFFF:
  // no entry), tags and impulses of its last solved rows
  DBuf<uint32_t> jw_n;
  DBuf<uint8_t> jw_tag;
  DBuf<float> jw_lam;
  // per tick: each joint's first row and row count, and its six XPBD multipliers
  DBuf<uint32_t> jr_cnt, jr_off;
  DBuf<float> jlam;
  uint32_t njr_ = 0;
  void drop_joint_warm_of(uint32_t body);      // drop_warm_of's joint part (world.rs:821-825)
  void restore_joint_warm(const SnapshotGpu* s);
  void filter_joint_warm_alive();              // restore_carried_state's joint part (world.rs:951-955)

  // ---- inspection
  const StepStatsHost& stats();
  void get_pairs(std::vector<uint64_t>& out);
  struct ContactOut { uint32_t a, b; float p[3], n[3]; float depth, impulse; uint32_t level; };
  void get_contacts(std::vector<ContactOut>& out);
  // The riftnet wire snapshot of the live bodies (riftphys-riftnet/src/wire.rs:36-53): sizes, and
  // the chunks packed into host_out when it is given (throws std::length_error past cap).
  void pack_snapshot(unsigned long long tick, unsigned long long epoch, uint8_t* host_out, size_t cap, size_t* bytes,
                     uint32_t* chunks);
  // World::raycast for n rays (queries.rs:50-116): rays8 per ray origin xyz, unit direction xyz,
  // max distance, ignored body index bits (0xFFFFFFFF: none); per ray hit point xyz with w the hit
  // body's id + 1 (0: no hit, 0xFFFFFFFF: the terrain) as bits, and normal xyz with w the fraction.
  // exact: World::raycast_exact (queries.rs:18-48), the true shapes instead of their AABBs
  void raycast_batch(uint32_t n, const float* rays8, float4* hit_pt, float4* hit_n, bool exact = false);
  // World::sweep_capsule for n queries (queries.rs:118-249): q12 per query from xyz, to xyz,
  // radius, half height, ignored body index bits, 3 words unused; out as raycast_batch's, the
  // normal's w -0.0 when the capsule started overlapping.
  void sweep_batch(uint32_t n, const float* q12, float4* hit_pt, float4* hit_n);
  uint32_t body_of_collider(uint32_t c) const { return h_col_body_[c]; }

  // ---- the kinematic player controller (world.rs:466-475; step.rs:544-639). The device holds
  // the controllers between ticks; the host copy is refreshed when the host reads or changes one.
  uint32_t add_player(const float pose[7], float radius, float height, float speed);
  uint32_t num_players() const { return (uint32_t)h_players_.size(); }
  void set_player_input(uint32_t i, const float dir[3]);
  void get_player(uint32_t i, float pose[7], bool* grounded);
  const std::vector<PlayerGpu>& players();   // the controllers as the device has them
  void set_players(const std::vector<PlayerGpu>& v);
  void run_players(float dt);                // World::update_players, at the start of a tick
  std::vector<PlayerGpu> h_players_;
  bool players_dev_newer_ = false;
  DBuf<PlayerGpu> players_d;
  DBuf<uint32_t> player_of_d;                // per body: its controller's index, or 0xFFFFFFFF

  // ---- the dynamic state as one host byte blob (layout in rphys_ext.h, rphys_ext_state_export)
  uint64_t state_bytes();
  void state_export(uint8_t* out);
  // throws std::invalid_argument when the blob does not fit this world's bodies and joints
  void state_import(const uint8_t* in, uint64_t bytes);

  // ---- rollback
  SnapshotGpu* snapshot_create();
  void snapshot_restore(const SnapshotGpu* s);
  void snapshot_restore_exact(const SnapshotGpu* s);  // every stored bit (rollback replay)
  static void snapshot_free(SnapshotGpu* s);

  cudaStream_t stream() const { return stream_; }
  int device() const { return dev_; }  // the device the world was created on (its stream's)
  // learned warm start: a model (owned by the caller) predicting each row's start, and logging of
  // the rows' features and converged impulses (its training data)
  WarmModel* model_ = nullptr;
  bool feat_log_ = false, pred_valid_ = false, pred_cold_only_ = false;
  void get_row_features(std::vector<float>& feats, std::vector<float>& targets);
  void get_row_predictions(std::vector<float>& pred4);
  // side streams the velocity solve forks onto (independent solve groups run concurrently)
  static constexpr int kAux = 7;  // one per single-island size bucket, one for the big islands
  cudaStream_t aux_[kAux] = {};
  cudaEvent_t ev_fork_ = nullptr, ev_join_[kAux] = {};
  // per-stage CUDA-event timing (totals since the last reset)
  void profile_enable(bool on);
  int profile_read(double* ms, uint64_t* calls, int cap);
  static const char* phase_name(int p);

 private:
  void upload_pair_table();
  void drop_warm_of(uint32_t b);
  void filter_warm(int mode, uint32_t body);  // mode 0: drop body, 1: keep alive keys only
  uint32_t read_u32(const uint32_t* dptr);

  // capacities and counts
  uint32_t cap_b_, cap_c_, nb_ = 0, ncol_ = 0;
  int dev_ = 0;
  cudaStream_t stream_ = nullptr;
  // host mirrors of static data
  std::vector<uint8_t> h_alive_;
  std::vector<uint32_t> h_col_body_, h_col_kind_, h_col_mat_;
  std::vector<float> h_col_dims_;
  std::vector<std::pair<std::pair<uint32_t, uint32_t>, PairPropsHost>> overrides_;
  f3 gravity_ = mk3(0.0f, -9.81f, 0.0f);
  uint64_t epoch_ = 0, rng_ = 0xC0FFEEull | 1ull, tick_ = 0;
  // heightfield
  bool has_hf_ = false;
  uint32_t hf_nx_ = 0, hf_nz_ = 0, hf_mat_ = 4;
  float hf_sx_ = 1, hf_sz_ = 1, hf_ox_ = 0, hf_oz_ = 0, hf_min_ = 0, hf_max_ = 0;
  DBuf<float> hf_h_;

 public:
  // solver configuration and device state (read by the pipeline in the .cu files)
  uint32_t iters_v_ = 20, iters_p_ = 20;
  float res_tol_ = 0.0f;
  uint32_t res_max_ = 0;
  DBuf<float4> pos, rot, lin, ang, last_lin;
  DBuf<float> inv_mass, inv_I;
  DBuf<uint8_t> dyn, awake, sleep_allowed, alive_d;
  DBuf<uint16_t> sleep_ticks;
  DBuf<uint32_t> col_body, col_kind, col_mat;
  DBuf<float4> col_dims;
  DBuf<float> pair_table;  // 14 x 14 x 5
  // warm cache
  DBuf<uint4> warm_key, warm_key2;
  DBuf<float4> warm_a, warm_b, warm_a2, warm_b2;  // a: la.xyz + jn, b: jt.xyz
  uint32_t n_warm = 0;
  // per-tick products kept for inspection
  uint32_t n_pairs = 0, n_contacts = 0;
  StepStatsHost st_;
  bool stats_dirty_ = false;
  bool levels_valid_ = false;
  struct Scratch;
  Scratch* s_ = nullptr;
  DBuf<uint32_t> d_stats;  // device-side counters
};

struct SnapshotGpu {
  uint64_t tick;
  uint32_t nb, cap, n_warm;
  DBuf<float4> pos, rot, lin, ang, last_lin;
  DBuf<uint8_t> awake;
  DBuf<uint16_t> ticks;
  DBuf<uint4> wk;
  DBuf<float4> wa, wb;
  uint32_t nj;
  DBuf<uint32_t> jw_n;
  DBuf<uint8_t> jw_tag;
  DBuf<float> jw_lam;
  std::vector<PlayerGpu> players;  // lib.rs:1696-1702
};

// MassProps::from_*_density (riftphys-geom/src/mass.rs:75-145); host side.
bool mass_from_density(uint32_t shape, const float dims[3], float density, float* inv_mass, float inertia[3]);
// pair_props with the built-in table (riftphys-materials/src/materials.rs:250-305)
PairPropsHost table_pair_props(uint32_t a, uint32_t b);
bool material_known(uint32_t id);

}  // namespace rp
