/* include/rphys_ext.h -- extensions to the v1 ABI. No v1 symbol changes; everything here is a
 * new export with the rphys_ext_ / rphys_batch_ prefix.
 *
 * The reference configures a world through its Rust World API, which the v1 C ABI does not
 * expose (the FFI ignores caller mass and friction: crates/riftphys-ffi/src/lib.rs:544-557,
 * 724-728). The setters below restate those World methods one for one so C hosts and the
 * benchmark scenes can reach them. Inspection calls return the step's intermediate products
 * (pair list, culled manifolds with their solver level, statistics) for parity checking.
 */
#pragma once

#include "riftphys_c.h"

#ifdef __cplusplus
extern "C" {
#endif

#define RPHYS_SHAPE_SPHERE  0u
#define RPHYS_SHAPE_BOX     1u
#define RPHYS_SHAPE_CAPSULE 2u

/* One body with one collider at its centre. Mass properties come from
 * MassProps::from_{sphere,box,capsule}_density(dims, density) (riftphys-geom/src/mass.rs:75-145). */
typedef struct RPhysBodyDescEx {
    RPhysIsometry pose;
    RPhysVelocity vel;
    uint32_t shape;        /* RPHYS_SHAPE_* */
    float dims[3];         /* sphere: r; box: hx, hy, hz; capsule: r, half_height */
    float density;         /* kg/m^3, dynamic bodies only */
    RPhysBodyType body_type;
    uint32_t material_id;  /* riftphys-materials MaterialId ordinal (0 = Default, 4 = Grit) */
    uint32_t sleep_allowed;/* World::set_body_sleep_allowed (world.rs:565-570) */
} RPhysBodyDescEx;

/* World::add_body + World::add_collider (riftphys-world/src/world/world.rs:595-622). Bodies get
 * consecutive 1-based ids; *out_first_id receives the first. */
RPhysResult rphys_ext_add_bodies(RPhysWorld* world, const RPhysBodyDescEx* descs, uint32_t n,
                                 uint32_t* out_first_id);

/* Contact properties for a material pair, either order (World::set_pair_props,
 * world.rs:975-979). Compliant (stiffness > 0) and patch-friction pairs are not supported. */
typedef struct RPhysPairProps { float mu_s, mu_k, restitution, stribeck_v; } RPhysPairProps;
RPhysResult rphys_ext_set_pair_props(RPhysWorld* world, uint32_t mat_a, uint32_t mat_b,
                                     const RPhysPairProps* props);

/* World::set_solver_iterations (world.rs:994-996): each is clamped to at least 1. */
RPhysResult rphys_ext_set_solver_iterations(RPhysWorld* world, uint32_t velocity, uint32_t position);

/* World::set_gravity (world.rs:560-563). */
RPhysResult rphys_ext_set_gravity(RPhysWorld* world, RPhysVec3 g);

/* HeightField::from_heights (riftphys-terrain/src/terrain.rs:24-50) from f32 samples, row-major
 * with x fastest (nx * nz values); replaces any terrain the world had. */
RPhysResult rphys_ext_set_heightfield_f32(RPhysWorld* world, uint32_t nx, uint32_t nz,
                                          float cell_x, float cell_z, float origin_x, float origin_z,
                                          const float* heights, uint32_t material_id);

/* Velocity-solve termination. tolerance <= 0: the reference's fixed iteration count. tolerance > 0:
 * sweep until the residual (largest |delta impulse| / effective mass over all rows in a sweep,
 * m/s) is <= tolerance, at most max_sweeps sweeps. */
RPhysResult rphys_ext_set_residual_mode(RPhysWorld* world, float tolerance, uint32_t max_sweeps);

/* Order of the order-dependent contact passes (warm-start application, velocity sweeps, ballistic
 * test, position projection). RPHYS_ORDER_SERIAL (default): the reference's serial order, through
 * its level schedule (crates/riftphys-world/src/world/solver.rs:621-642), bit for bit.
 * RPHYS_ORDER_COLOURED (an extension; the reference has no such order): each solve island is
 * coloured by first fit in level order -- a row takes the smallest colour no already coloured row
 * writing one of its bodies holds, at most 128 per body (an island needing more keeps its levels) --
 * and the passes run colour by colour. Fewer, wider steps than the levels; the Gauss-Seidel updates
 * are reordered, so results differ from the serial order's (they match the CPU restatement's
 * coloured order bit for bit). Worlds with joints keep the serial order. */
#define RPHYS_ORDER_SERIAL   0u
#define RPHYS_ORDER_COLOURED 1u
RPhysResult rphys_ext_set_solve_order(RPhysWorld* world, uint32_t order);

/* Launch shapes of the velocity solve (an extension; no reference counterpart). None changes a
 * result bit: islands are independent, and so are the rows of one level or colour. group_rows:
 * islands of at most this many rows are packed into shared solve groups (8, 16, 32, 64 or 128); packed_threads:
 * threads of a packed group's block (32, 64 or 128); island_threads: threads of a single island's
 * block (32, 64, 128 or 256). Defaults are the autotuner's choice for the terrain workload (bench.py
 * --autotune, recorded in riftphys-rust_b200/tuning.json). Other values give RPHYS_ERR_BAD_ARG. The
 * CPU restatement stores and returns them. */
typedef struct RPhysTuning { uint32_t group_rows, packed_threads, island_threads; } RPhysTuning;
RPhysResult rphys_ext_set_tuning(RPhysWorld* world, const RPhysTuning* tuning);
RPhysResult rphys_ext_get_tuning(const RPhysWorld* world, RPhysTuning* out);

/* Runs n ticks of dt (each one World::step) with a single completion wait at the end. */
RPhysResult rphys_ext_step_n(RPhysWorld* world, float dt, uint32_t n);

#define RPHYS_STATERR_NONFINITE_AABB  1u   /* an AABB with a non-finite bound beyond min.x */
#define RPHYS_STATERR_CAPACITY        2u   /* a per-step buffer overflowed; results invalid */
#define RPHYS_STATERR_WAIT_TIMEOUT    4u   /* a bounded device wait gave up */

typedef struct RPhysStepStats {
    uint32_t pairs;          /* broadphase pairs (StepStats::pairs_tested) */
    uint32_t contacts;       /* culled contact points (StepStats::contacts) */
    uint32_t islands;        /* StepStats::islands */
    uint32_t levels;         /* levels of the solve schedule (joint rows, then contact rows) */
    uint32_t max_batch;      /* largest level (World::last_max_batch().0 without joints) */
    uint32_t warm_matched;   /* contacts started warm (World::warm_matched) */
    uint32_t sweeps;         /* velocity sweeps run in the last tick */
    uint32_t bounce_rows;    /* rows the W6 bounce pass solved at their time of impact (BounceStats::toi_rows) */
    uint32_t warm_entries;   /* entries in the warm-start cache (World::warm_contacts) */
    uint32_t sleeping;       /* bodies asleep (World::num_sleeping) */
    uint32_t error_flags;    /* RPHYS_STATERR_* */
    float residual;          /* residual of the last velocity sweep (m/s) */
    uint32_t row_sweeps;     /* velocity row updates run in the last tick (rows x sweeps) */
    uint32_t rows_scheduled; /* contact rows with a movable body, and joint rows, in the last tick */
    /* how the last tick's velocity solve was split (0 from the CPU restatement): solve groups whose
     * rows and bodies fit in on-chip shared memory, groups solved over global memory, and the
     * largest group */
    uint32_t groups_shared, groups_global, max_group_rows, max_group_bodies;
    uint32_t islands_capped; /* residual mode: solve islands still above the tolerance at the sweep cap */
    uint32_t pred_used;      /* rows whose warm start came from the learned prediction */
    uint32_t rows_capped;    /* residual mode: rows of the islands counted in islands_capped */
    /* solve islands by the residual of their last sweep (m/s): <= 1e-4, <= 1e-3, <= 1e-2, <= 1e-1,
     * <= 1, above 1 */
    uint32_t res_hist[6];
} RPhysStepStats;
RPhysResult rphys_ext_get_stats(const RPhysWorld* world, RPhysStepStats* out);

/* Last tick's broadphase pairs as (i, j) collider indices, i < j, ascending. */
RPhysResult rphys_ext_get_pairs(const RPhysWorld* world, uint32_t* out_ij, uint32_t cap_pairs,
                                uint32_t* out_count);

/* Last tick's culled, oriented contacts in solve order, with their solver level
 * (0xFFFFFFFF: no movable body, not scheduled). */
typedef struct RPhysContactRecord {
    uint32_t a_collider, b_collider;   /* b = 0xFFFFFFFF for terrain */
    RPhysVec3 point, normal;
    float depth, impulse;
    uint32_t level;
    uint32_t pad;
} RPhysContactRecord;
RPhysResult rphys_ext_get_contact_records(const RPhysWorld* world, RPhysContactRecord* out,
                                          uint32_t cap, uint32_t* out_count);

/* Raw state of bodies [first, first + count) (internal 0-based indices): 13 floats each,
 * pos xyz, rot xyzw, lin xyz, ang xyz. */
RPhysResult rphys_ext_get_body_states(const RPhysWorld* world, uint32_t first, uint32_t count,
                                      float* out13);

/* Per-stage timing with CUDA events recorded on the world's stream around each stage of the tick
 * (on: also waits for each tick to finish). read: totals in ms and tick counts since enabling;
 * returns the number of stages; names from rphys_ext_profile_stage_name. */
RPhysResult rphys_ext_profile_enable(RPhysWorld* world, uint32_t on);
RPhysResult rphys_ext_profile_read(const RPhysWorld* world, double* ms, uint64_t* ticks, uint32_t cap,
                                   uint32_t* out_stages);
const char* rphys_ext_profile_stage_name(uint32_t stage);

/* The CUDA stream every kernel of this world runs on (a cudaStream_t), for callers that time or
 * order their own work against the tick. 0 from a library without a device. */
RPhysResult rphys_ext_stream_handle(const RPhysWorld* world, uint64_t* out_stream);

/* Device kernels this library has launched since it was loaded (all worlds): every launch site
 * counts its kernels, and each device-wide sort, scan or select counts the kernels it runs. */
RPhysResult rphys_ext_launch_count(uint64_t* out_launches);

/* ---- Batched worlds (no counterpart in the reference, which steps one World per call).
 * Many independent worlds live in one RPhysWorld and are stepped together by rphys_world_step_ex
 * / rphys_ext_step_n: every kernel of the tick covers all of them, bodies of different worlds never
 * pair, and each world's results are bit-identical to stepping it alone. Worlds are appended in
 * order, each with all its bodies in one call; the first call must be on an empty RPhysWorld.
 * Ids stay global 1-based (a world's bodies are one contiguous run); gravity, pair properties,
 * iterations, residual mode and a heightfield (if set) are shared. Snapshot and restore cover the
 * whole batch (rollback of every world at once). */
RPhysResult rphys_ext_batch_add_world(RPhysWorld* world, const RPhysBodyDescEx* descs, uint32_t count,
                                      uint32_t* out_world, uint32_t* out_first_id);
RPhysResult rphys_ext_batch_num_worlds(const RPhysWorld* world, uint32_t* out_count);
RPhysResult rphys_ext_batch_world_range(const RPhysWorld* world, uint32_t world_index, uint32_t* out_first_id,
                                        uint32_t* out_count);
/* Restores every bit a snapshot holds (poses, velocities, carried state, warm-start cache) as a
 * World clone would, where rphys_world_snapshot_restore follows the reference FFI
 * (lib.rs:1754-1793) and re-injects poses through set_pose, which renormalises rotations, so a
 * replay after it can differ in the last bits. For rollback windows whose re-simulation must
 * reproduce the first pass's hashes (no counterpart in the reference FFI). The body set must be
 * the snapshot's: RPHYS_ERR_BAD_ARG otherwise. */
RPhysResult rphys_ext_snapshot_restore_exact(RPhysWorld* world, const RPhysWorldSnapshot* snapshot);

/* Per-world tick hashes: world k's digest equals rphys_world_get_step_hash of a world created with
 * capacity = its body count and holding only its bodies. */
RPhysResult rphys_ext_batch_get_hashes(const RPhysWorld* world, uint32_t first_world, uint32_t count,
                                       RPhysHash32* out_hashes);

/* ---- The learned warm start's model (no counterpart in the reference). An MLP 24 -> 128 -> 128 ->
 * 128 -> 3 with SiLU, bf16 weights and activations with f32 accumulation on the tensor cores,
 * trained on the GPU with Adam on f32 master weights. Inputs: 24 f32 features per contact row (the
 * layout rphys_ext_get_row_features writes); outputs: the row's impulse (normal, two friction
 * components) in units of the row's effective mass x 9.81 / 60. Weights are one f32 array of
 * rphys_ext_model_num_params() values (W1 [128 x 32], b1, W2 [128 x 128], b2, W3, b3, W4 [16 x 128],
 * b4 [16]; the padding columns of W1 and rows of W4 stay 0). */
typedef struct RPhysWarmModel RPhysWarmModel;
RPhysWarmModel* rphys_ext_model_create(uint64_t seed);
void rphys_ext_model_destroy(RPhysWarmModel* model);
uint32_t rphys_ext_model_num_params(void);
RPhysResult rphys_ext_model_get_weights(const RPhysWarmModel* model, float* out, uint32_t count);
RPhysResult rphys_ext_model_set_weights(RPhysWarmModel* model, const float* in, uint32_t count);
RPhysResult rphys_ext_model_predict(RPhysWarmModel* model, const float* feats24, uint32_t rows, float* out3);
/* The same with device pointers (24 floats in, 3 out per row) on the given CUDA stream (0: the
 * model's own); returns after the predictions are written. */
RPhysResult rphys_ext_model_predict_device(RPhysWarmModel* model, const float* dev_feats24, uint32_t rows, float* dev_out3,
                                           uint64_t cuda_stream);
/* One forward/backward pass (mean squared error over the 3 outputs): gradients of every weight. */
RPhysResult rphys_ext_model_gradients(RPhysWarmModel* model, const float* feats24, const float* targets3, uint32_t rows,
                                      float* out_grads, float* out_loss);
/* `epochs` passes of mini-batch Adam over the rows in order; returns the last epoch's mean loss. */
RPhysResult rphys_ext_model_train(RPhysWarmModel* model, const float* feats24, const float* targets3, uint32_t rows,
                                  uint32_t epochs, uint32_t batch, float learning_rate, float* out_loss);

/* The learned warm start in a world (no counterpart in the reference). With a model set (it must
 * outlive its use; NULL switches it off), every tick computes each contact row's features and the
 * model's predicted impulse; at the row's place in the warm-start order the solver tries both the
 * previous tick's impulse (or none) and the prediction on copies of the two bodies and keeps the
 * one that leaves the smaller normal velocity error, so a prediction that would start the row
 * worse falls back to the reference warm start. Counted in RPhysStepStats.pred_used. The
 * predictions are computed on the tensor cores and are deterministic, so replays and hashes are. */
RPhysResult rphys_ext_set_warm_model(RPhysWorld* world, RPhysWarmModel* model);
/* cold_only = 1: offer predictions only to rows the previous tick's cache has no impulse for (new
 * contacts); 0 (the default): to every row. */
RPhysResult rphys_ext_set_warm_policy(RPhysWorld* world, uint32_t cold_only);
/* Training data: with logging on, the last tick's feature rows (24 floats) and converged impulses
 * (3 floats, the model's output unit) of the contacts with a movable body, in contact order. */
RPhysResult rphys_ext_set_feature_logging(RPhysWorld* world, uint32_t on);
RPhysResult rphys_ext_get_row_features(const RPhysWorld* world, float* out_feats24, float* out_targets3, uint32_t cap_rows,
                                       uint32_t* out_rows);
/* The predictions the last tick offered, per contact in contact order: 4 floats (normal, friction 1,
 * friction 2, 1) or zeros where none was offered. */
RPhysResult rphys_ext_get_row_predictions(const RPhysWorld* world, float* out4, uint32_t cap_contacts, uint32_t* out_count);

/* D6 joints: World::add_ball_joint / add_hinge_joint (riftphys-world/src/world/world.rs:718-719;
 * Joints::add_ball / add_hinge, riftphys-articulation/src/bodies.rs:326-338). frame_a / frame_b
 * place the joint frame in body A's / body B's frame. A ball locks the three translations and
 * leaves rotation free; a hinge also locks the two rotations other than hinge_axis (0, 1, 2 = x,
 * y, z of frame A). Bodies joined by a joint never collide with each other (step.rs:85-102).
 * Joint ids are 0-based, in creation order; *out_first_id receives the first. Body ids as
 * everywhere (1-based, live); body_a != body_b; frames finite. In a batch (rphys_ext_batch_*), a
 * joint joins two bodies of one world and joints come in world order (each world's joints one
 * id range, hashed by rphys_ext_batch_get_hashes with ids from 0). All-or-nothing: a bad
 * descriptor adds none. */
#define RPHYS_JOINT_BALL  0u
#define RPHYS_JOINT_HINGE 1u
#define RPHYS_JOINT_D6    2u   /* World::add_d6_joint with every axis enabled (locked), no stored hinge axis */
typedef struct RPhysJointDesc {
    uint32_t kind;         /* RPHYS_JOINT_* */
    uint32_t hinge_axis;   /* RPHYS_JOINT_HINGE only */
    uint32_t body_a, body_b;
    RPhysIsometry frame_a, frame_b;
} RPhysJointDesc;
RPhysResult rphys_ext_add_joints(RPhysWorld* world, const RPhysJointDesc* descs, uint32_t n, uint32_t* out_first_id);
/* World::add_distance_joint / add_distance_joint_at + set_distance_damping (world.rs:537-552;
 * bodies.rs:273-305): body_b's anchor held at `rest` from body_a's (anchors in each body's frame),
 * compliance in m/N (0 = rigid, else a spring at position level), damping in N s/m along the rod.
 * Both anchors zero and no damping is the original centre-to-centre rod (its own velocity row,
 * solver.rs:793-817); otherwise the anchored rows (the rod passes torque through its lever arms).
 * Joint ids are shared with rphys_ext_add_joints; bodies so joined no longer collide. Finite
 * values, compliance and damping >= 0; all-or-nothing over the array. */
typedef struct RPhysDistanceJointDesc {
    uint32_t body_a, body_b;
    RPhysVec3 anchor_a, anchor_b;
    float rest, compliance, damping;
} RPhysDistanceJointDesc;
RPhysResult rphys_ext_add_distance_joints(RPhysWorld* world, const RPhysDistanceJointDesc* descs, uint32_t n,
                                          uint32_t* out_first_id);
/* Joints::set_d6_limit_t (angular = 0) / set_d6_limit_r (angular = 1) (bodies.rs:367-391): with
 * enabled, the axis becomes a limited row on [lo, hi] (metres along frame A's axis, or radians:
 * the twist angle on a hinge's own axis, 2 sin(angle / 2) about the other axes); a limit on a
 * rotational axis other than a hinge's own makes the joint no longer a hinge. enabled = 0 clears
 * the limit and leaves the axis as it was. lo <= hi, both finite. */
RPhysResult rphys_ext_set_joint_limit(RPhysWorld* world, uint32_t joint, uint32_t angular, uint32_t axis,
                                      uint32_t enabled, float lo, float hi);
/* The same for many limits at once, applied in array order; all-or-nothing. */
typedef struct RPhysJointLimit {
    uint32_t joint, angular, axis, enabled;
    float lo, hi;
} RPhysJointLimit;
RPhysResult rphys_ext_set_joint_limits(RPhysWorld* world, const RPhysJointLimit* limits, uint32_t n);
RPhysResult rphys_ext_num_joints(const RPhysWorld* world, uint32_t* out_count);

/* D6Axis.enabled and .compliance of one axis (m/N or rad/(N m); 0 = rigid), as a D6Joint built for
 * World::add_d6_joint sets them (riftphys-articulation/src/bodies.rs:80-108). A compliant axis has
 * no velocity row and acts as an XPBD spring at position level; a rotational axis whose compliance
 * is at least 100x each other enabled one makes the joint a sprung hinge about it
 * (d6_hinge_axis, bodies.rs:891-901). compliance finite and >= 0. */
RPhysResult rphys_ext_set_joint_axis(RPhysWorld* world, uint32_t joint, uint32_t angular, uint32_t axis,
                                     uint32_t enabled, float compliance);
/* Joints::set_d6_drive_t / set_d6_drive_r (bodies.rs:354-366); drive = NULL clears it. A position
 * drive (vel_mode 0) holds the axis at target (clamped into its limit) at position level; a
 * velocity drive is a motor row driving the relative velocity to target with at most
 * |max_impulse| per tick, and bodies of a joint with a rotational velocity drive keep the angular
 * velocity the solve gave them (step.rs:352-366). Setting one enables the axis. Finite values. */
typedef struct RPhysJointDrive { float target, kp, kd, max_impulse; uint32_t vel_mode; } RPhysJointDrive;
RPhysResult rphys_ext_set_joint_drive(RPhysWorld* world, uint32_t joint, uint32_t angular, uint32_t axis,
                                      const RPhysJointDrive* drive);
/* Joints::set_d6_damping (bodies.rs:376-383): viscous damping (N m s/rad or N s/m; an implicit
 * velocity row, or XPBD's damping term on a compliant unlimited row) and Coulomb friction (N m or
 * N: at most friction x dt of impulse per tick) on one axis, free axes too. Negative or non-finite
 * values become 0, as in the reference. */
RPhysResult rphys_ext_set_joint_damping(RPhysWorld* world, uint32_t joint, uint32_t angular, uint32_t axis,
                                        float damping, float friction);

/* The riftnet wire snapshot (riftphys-riftnet/src/wire.rs:1-53): every live body, in id order, as
 * a NetEnt {u32 id (the FFI body id); f32 px py pz, qx qy qz qw, sx sy sz; u32 kind} of 48 bytes
 * -- kind 1 sphere (scale r r r), 2 box (the half extents), 3 capsule along y (r, (hh + r) / 2, r)
 * as wire.rs:22-23 defines -- 25 to a chunk (MAX_PAYLOAD 1200 bytes) behind a 32-byte NetHdr
 * {u32 magic 0x30535052; u16 ver 2; u8 kind 1; u8 flags 0; u64 tick; u64 epoch; u16 total;
 * u16 index; u32 payload_len}, the chunks back to back in out (chunk c at c x 1232 bytes): what
 * pack_snapshot(tick, epoch, ents) returns, one datagram per chunk. Packed on the device; out
 * NULL only reports the sizes (out_bytes, out_chunks). total is the chunk count as u16, as in the
 * reference. RPHYS_ERR_CAPACITY when out_cap is smaller than the snapshot. */
#define RPHYS_WIRE_MAGIC 0x30535052u
#define RPHYS_WIRE_HEADER_BYTES 32u
#define RPHYS_WIRE_ENTITY_BYTES 48u
#define RPHYS_WIRE_ENTITIES_PER_CHUNK 25u
RPhysResult rphys_ext_pack_snapshot(RPhysWorld* world, uint64_t tick, uint64_t epoch, uint8_t* out, uint64_t out_cap,
                                    uint64_t* out_bytes, uint32_t* out_chunks);

/* rphys_world_raycast for n rays at once, one device block per ray; every query checked first
 * (all-or-nothing), then out[i] as rphys_world_raycast would write it for queries[i]. */
RPhysResult rphys_ext_raycast_batch(const RPhysWorld* world, const RPhysRayQuery* queries, uint32_t n,
                                    RPhysRayHit* out);
/* World::raycast_exact (crates/riftphys-world/src/world/queries.rs:18-48; ray_shape,
 * crates/riftphys-geom/src/raycast.rs:13-130) for n rays: the true shapes (rotated boxes, spheres,
 * capsules, terrain triangles) instead of the colliders' AABBs. Skips ignore_body (the reference's
 * skip predicate, for one body). Checked and normalised as rphys_world_raycast; normals face the
 * ray, and a ray starting inside a solid hits at fraction 0 with normal -dir. */
RPhysResult rphys_ext_raycast_exact_batch(const RPhysWorld* world, const RPhysRayQuery* queries, uint32_t n,
                                          RPhysRayHit* out);

/* The world's dynamic state as one flat little-endian byte blob (no counterpart in the
 * reference, whose World clone, crates/riftphys-world/src/world/world.rs:912-961, stays inside one
 * process). It holds every stored bit a tick reads that the world's set-up does not fix: the tick,
 * epoch and rng state; per body its pose, velocities and last linear velocity; the sleep state at
 * the world's capacity; the contact and joint warm-start caches. Importing it into a world built
 * with the same bodies, joints and settings (in this library or in any library with this ABI, a CPU
 * world included) makes that world's next ticks bit-identical to the exporter's. Layout: a 48-byte
 * header ("RPS1", version 1, tick, epoch, rng as u64; bodies, capacity, warm entries, joints as u32),
 * 64 bytes per body (pos xyz, rot xyzw, lin xyz, ang xyz, last linear velocity xyz as f32), one
 * alive byte per body, one awake byte per capacity slot, then one u16 sleep counter per slot,
 * 44 bytes per warm entry (key: body a, body b or 0xFFFFFFFF, ordinals a and b as u32; anchor xyz,
 * normal impulse, friction impulse xyz as f32), 164 bytes per joint (cached row count u32 with
 * 0xFFFFFFFF for none, 32 row tags u8, 32 impulses f32). With out NULL, *out_bytes receives the size;
 * a buffer below it gives RPHYS_ERR_CAPACITY. Worlds with players have no blob (RPHYS_ERR_BAD_ARG). */
RPhysResult rphys_ext_state_export(const RPhysWorld* world, uint8_t* out, uint64_t out_cap, uint64_t* out_bytes);
/* Loads a blob of rphys_ext_state_export. RPHYS_ERR_BAD_ARG, with nothing changed, when its body
 * count, capacity, joint count or live bodies differ from this world's, or its size does not match
 * its counts. */
RPhysResult rphys_ext_state_import(RPhysWorld* world, const uint8_t* in, uint64_t bytes);

/* rphys_world_get_step_hash without any device allocation (no counterpart in the reference, whose
 * hash runs on the CPU). For hosts that hash every tick from a thread that must not allocate:
 * cudaMalloc and cudaFree can wait for all work on the device and their memory use varies with the
 * world, while this call's scratch is one fixed array (about 16.5 MB per device) reserved when the
 * library is loaded. The digest is identical to rphys_world_get_step_hash's. Limits: a state
 * stream of at most 12 MiB (56 + 12 bytes per body, 3 bytes per body of capacity, up to 48 bytes
 * per warm-start entry), at most 262144 warm-start entries and 65536 joints; a larger world returns
 * RPHYS_ERR_CAPACITY with the sizes in rphys_last_error_message and runs nothing on the device.
 * Joints added or changed since the last step are not uploaded by this call (the next step does
 * that): their warm-cache entries do not exist yet, so the digest is unchanged by them. The call
 * runs on the device the world was created on, whatever device the calling thread has current.
 * The first call on each device looks up the array's address there (device setup): make it once
 * before the real-time loop. The array is shared by every world on a device, so calls are
 * serialised inside the library; each returns after its device work finished. */
RPhysResult rphys_ext_world_step_hash_noalloc(const RPhysWorld* world, RPhysHash32* out_hash);

#ifdef __cplusplus
}
#endif
