/* include/riftphys_c.h -- the drop-in boundary: the reference's C ABI, version 1.
 *
 * Every declaration restates crates/riftphys-ffi/src/riftphys_c.h (ABI v1) with identical
 * names, layouts and error codes, so a host compiled against the reference header links
 * against librphys_gpu.so unchanged. The one addition is the declaration of
 * RPhysContactEvent, which the reference header uses (riftphys_c.h:248-253) but never
 * declares; its layout is the Rust definition at crates/riftphys-ffi/src/lib.rs:107-115.
 *
 * Each entry point below cites the reference function it replaces (file:line in
 * crates/riftphys-ffi/src/lib.rs). Ray casts, capsule sweeps and the kinematic player controller
 * are exported and run on the device.
 */
#pragma once

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ===================== ABI VERSION ===================== */
#define RPHYS_ABI_VERSION 1u
uint32_t    rphys_get_abi_version(void);        /* lib.rs:85-88 */
const char* rphys_get_build_id(void);           /* lib.rs:90-95 */

/* ===================== ABI TYPES ===================== */
typedef uint32_t RPhysBool;
#define RPHYS_FALSE 0u
#define RPHYS_TRUE  1u

typedef uint32_t RPhysResult;
#define RPHYS_OK             0u
#define RPHYS_ERR_NULL       1u
#define RPHYS_ERR_INVALID_ID 2u
#define RPHYS_ERR_CAPACITY   3u
#define RPHYS_ERR_BAD_ARG    4u
#define RPHYS_ERR_INTERNAL   0x80000000u

#define RPHYS_INVALID_BODY_ID 0u
#define RPHYS_TERRAIN_BODY_ID 0xFFFFFFFFu

/* Thread-local message of the last failed call on this thread (lib.rs:73-83). */
const char* rphys_last_error_message(void);

typedef struct RPhysWorld RPhysWorld;

/* ===================== POD TYPES ===================== */
typedef struct RPhysVec3 { float x, y, z; } RPhysVec3;
typedef struct RPhysQuat { float x, y, z, w; } RPhysQuat;
typedef struct RPhysIsometry { RPhysVec3 pos; RPhysQuat rot; } RPhysIsometry;
typedef struct RPhysVelocity { RPhysVec3 lin; RPhysVec3 ang; } RPhysVelocity;
typedef struct RPhysMaterial { float mu_static; float mu_dynamic; float restitution; } RPhysMaterial;

typedef uint32_t RPhysBodyType;
#define RPHYS_BODY_STATIC  0u
#define RPHYS_BODY_DYNAMIC 1u

typedef struct RPhysCapsuleBodyDesc {
    RPhysIsometry pose; RPhysVelocity vel;
    float radius; float half_height; float mass;
    RPhysBodyType body_type; RPhysMaterial material; uint32_t user_tag;
} RPhysCapsuleBodyDesc;

typedef struct RPhysBoxBodyDesc {
    RPhysIsometry pose; RPhysVelocity vel;
    float hx, hy, hz; float mass;
    RPhysBodyType body_type; RPhysMaterial material; uint32_t user_tag;
} RPhysBoxBodyDesc;

typedef struct RPhysSphereBodyDesc {
    RPhysIsometry pose; RPhysVelocity vel;
    float radius; float mass;
    RPhysBodyType body_type; RPhysMaterial material; uint32_t user_tag;
} RPhysSphereBodyDesc;

#define RPHYS_STEP_HASH_BYTES 32
typedef struct RPhysHash32 { uint8_t bytes[RPHYS_STEP_HASH_BYTES]; } RPhysHash32;

typedef struct RPhysStepParams {
    uint32_t size_bytes;   /* must be >= sizeof(RPhysStepParams) */
    uint32_t flags;        /* reserved, ignored (lib.rs:1147-1148) */
    uint32_t substeps;     /* must be > 0 */
    uint32_t solver_iters; /* ignored, as in the reference (lib.rs:1147) */
    float    dt;           /* finite and >= 0 */
} RPhysStepParams;

/* Declared here because the reference header omits it (lib.rs:107-115). 36 bytes. */
typedef struct RPhysContactEvent {
    uint32_t body_id_a;
    uint32_t body_id_b;   /* RPHYS_TERRAIN_BODY_ID for heightfield contacts */
    RPhysVec3 position;
    RPhysVec3 normal;
    float impulse;        /* accumulated normal impulse of the last step */
} RPhysContactEvent;

typedef struct RPhysHeightfieldDesc {
    uint32_t size_bytes; uint32_t flags;
    uint32_t width; uint32_t height; uint32_t row_stride;
    float cell_size_x; float cell_size_z;
    float height_scale; float height_offset;
    const int16_t* heights;
} RPhysHeightfieldDesc;

/* ===================== QUERIES ===================== */
typedef struct RPhysRayQuery {
    RPhysVec3 origin;
    RPhysVec3 dir;          /* need not be normalised; zero is a miss */
    float max_distance;     /* <= 0: a miss */
    uint32_t ignore_body;   /* 1-based; 0 = none; the terrain sentinel is invalid here */
} RPhysRayQuery;
typedef struct RPhysRayHit {
    RPhysBool hit;
    uint32_t  body_id;      /* 1-based; 0 = none; RPHYS_TERRAIN_BODY_ID for the heightfield */
    float     fraction;     /* distance / max_distance, in [0, 1] */
    RPhysVec3 point;
    RPhysVec3 normal;
} RPhysRayHit;
/* World::raycast (riftphys-world/src/world/queries.rs:50-116; lib.rs:1271-1346): the nearest of the
 * colliders' AABBs and the heightfield's triangles along the ray; a miss is hit 0, body 0, fraction
 * 1, point 0, normal +Y. */
RPhysResult rphys_world_raycast(const RPhysWorld* world, const RPhysRayQuery* query, RPhysRayHit* out_hit);
typedef struct RPhysCapsuleSweepQuery {
    RPhysVec3 from;
    RPhysVec3 to;
    float radius;           /* finite, > 0 */
    float half_height;      /* finite, >= 0; the capsule is upright (local y) */
    uint32_t ignore_body;   /* 1-based; 0 = none; the terrain sentinel is invalid here */
} RPhysCapsuleSweepQuery;
typedef struct RPhysCapsuleSweepHit {
    RPhysBool hit;
    uint32_t  body_id;      /* 1-based; 0 = none; RPHYS_TERRAIN_BODY_ID for the heightfield */
    float     fraction;     /* of the way from -> to, in [0, 1]; 0 when it started overlapping */
    RPhysBool started_overlapping;
    RPhysVec3 point;
    RPhysVec3 normal;
} RPhysCapsuleSweepHit;
/* World::sweep_capsule (queries.rs:118-249; lib.rs:1349-1411): overlap at from first (the
 * narrowphase against colliders, then terrain triangles), else the capsule's tip and base spheres
 * swept against the colliders' and the terrain triangles' AABBs. */
RPhysResult rphys_world_capsule_sweep(const RPhysWorld* world, const RPhysCapsuleSweepQuery* query,
                                      RPhysCapsuleSweepHit* out_hit);

/* ===================== KINEMATIC PLAYER CONTROLLER ===================== */
typedef struct RPhysPlayerDesc {
    RPhysIsometry start_pose;
    float radius;           /* finite, > 0 */
    float height;           /* finite, > 0; the capsule's half height is height / 2 */
    float speed;
} RPhysPlayerDesc;
/* World::add_player (world.rs:466-475; lib.rs:1580-1627): a static body with a capsule collider of
 * radius 0.4 and half height 0.9, whatever the desc's size, which the controller's sweeps use.
 * Takes one body and one collider of the world's capacity. Returns a 0-based player index. */
RPhysResult rphys_add_player(RPhysWorld* world, const RPhysPlayerDesc* desc, uint32_t* out_player_idx);
/* The player's move direction for the next ticks (lib.rs:1668-1693); any length, normalised by the
 * step. */
RPhysResult rphys_player_set_input(RPhysWorld* world, uint32_t player_idx, RPhysVec3 move_dir);
/* The player body's pose and whether the last tick's slide found a floor (lib.rs:1629-1666). */
RPhysResult rphys_player_get_pose(const RPhysWorld* world, uint32_t player_idx, RPhysIsometry* out_pose,
                                  RPhysBool* out_grounded);

/* ===================== API ===================== */
RPhysResult rphys_world_set_heightfield_i16(RPhysWorld* world, const RPhysHeightfieldDesc* hf,
                                            float origin_x, float origin_z, float y_offset);  /* lib.rs:1420-1496 */
RPhysResult rphys_world_set_heightfield_raw32_square(RPhysWorld* world, const uint8_t* bytes, uint32_t bytes_len,
                                                     float world_size_x, float world_size_z,
                                                     float origin_x, float origin_z, float y_offset); /* lib.rs:1498-1548 */
RPhysResult rphys_world_clear_heightfield(RPhysWorld* world);                       /* lib.rs:1550-1566 */

RPhysWorld* rphys_world_create(uint32_t max_bodies, uint32_t max_colliders);       /* lib.rs:608-632 */
void        rphys_world_destroy(RPhysWorld* world);                                /* lib.rs:634-639 */
RPhysResult rphys_world_set_epoch(RPhysWorld* world, uint64_t epoch);              /* lib.rs:641-656 */
RPhysResult rphys_world_set_rng_seed(RPhysWorld* world, uint64_t seed);            /* lib.rs:658-673 */

RPhysResult rphys_add_capsule_body(RPhysWorld* world, const RPhysCapsuleBodyDesc* desc, uint32_t* out_body_id); /* lib.rs:677-751 */
RPhysResult rphys_add_box_body(RPhysWorld* world, const RPhysBoxBodyDesc* desc, uint32_t* out_body_id);         /* lib.rs:753-830 */
RPhysResult rphys_add_sphere_body(RPhysWorld* world, const RPhysSphereBodyDesc* desc, uint32_t* out_body_id);   /* lib.rs:832-900 */
RPhysResult rphys_body_remove(RPhysWorld* world, uint32_t body_id);                                               /* lib.rs:902-927 */

RPhysResult rphys_body_get_pose(const RPhysWorld* world, uint32_t body_id, RPhysIsometry* out_pose);   /* lib.rs:931-962 */
RPhysResult rphys_body_set_pose(RPhysWorld* world, uint32_t body_id, const RPhysIsometry* pose);        /* lib.rs:964-995 */
RPhysResult rphys_body_get_velocity(const RPhysWorld* world, uint32_t body_id, RPhysVelocity* out_vel); /* lib.rs:1002-1035 */
RPhysResult rphys_body_set_velocity(RPhysWorld* world, uint32_t body_id, const RPhysVelocity* vel);     /* lib.rs:1037-1067 */
RPhysResult rphys_body_apply_impulse(RPhysWorld* world, uint32_t body_id, RPhysVec3 impulse);         /* lib.rs:1069-1097 */

RPhysResult rphys_world_step_ex(RPhysWorld* world, const RPhysStepParams* p);  /* lib.rs:1101-1152 */
RPhysResult rphys_world_step(RPhysWorld* world, float dt);                     /* lib.rs:1154-1164 */

RPhysResult rphys_world_tick_index(const RPhysWorld* world, uint64_t* out_tick);               /* lib.rs:1168-1190 */
RPhysResult rphys_world_num_bodies(const RPhysWorld* world, uint32_t* out_num);                /* lib.rs:1192-1214 */
RPhysResult rphys_world_get_step_hash(const RPhysWorld* world, RPhysHash32* out_hash);         /* lib.rs:1216-1243 */
RPhysResult rphys_world_step_and_hash(RPhysWorld* world, float dt, RPhysHash32* out_hash);     /* lib.rs:1245-1262 */

RPhysResult rphys_last_error_copy(char* dst, uint32_t cap, uint32_t* out_len);                 /* lib.rs:560-604 */

RPhysResult rphys_world_get_contacts(const RPhysWorld* world, RPhysContactEvent* out_buffer,
                                     uint32_t buffer_capacity, uint32_t* out_count);           /* lib.rs:1801-1877 */

typedef struct RPhysWorldSnapshot RPhysWorldSnapshot;
RPhysWorldSnapshot* rphys_world_snapshot_create(const RPhysWorld* world);                      /* lib.rs:1707-1752 */
RPhysResult         rphys_world_snapshot_restore(RPhysWorld* world, const RPhysWorldSnapshot* snapshot); /* lib.rs:1754-1793 */
void                rphys_world_snapshot_free(RPhysWorldSnapshot* snapshot);                   /* lib.rs:1795-1800 */

#ifdef __cplusplus
}
#endif
