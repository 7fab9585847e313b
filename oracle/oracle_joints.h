// oracle/oracle_joints.h -- TEST INFRASTRUCTURE (the oracle): D6 joint rows and the joint
// position solve, restated from riftphys-world/src/world/solver.rs:264-424 and
// riftphys-articulation/src/bodies.rs:422-922. Only the oracle's World::step uses it.
#pragma once
#include <cstdint>
#include <vector>

#include "oracle_world.h"

namespace orc {

// JointRow (solver.rs:264-288): gamma = 1 / (damping dt) on a damper row, 0 on the others.
struct JRow {
  uint32_t a, b, joint;
  bool angular;
  V3 u, ra, rb;
  float wa, wb, m_eff, target, lam_min, lam_max;
  uint8_t tag;
  float gamma = 0.0f;
  uint8_t idx = 0, cnt = 0;  // index in its joint's rows; the joint's row count (on its first row)
  // the original distance row (solver.rs:793-817): impulse -(v_rel + bias) / inv_sum along u on
  // the linear velocities, bias = (len - rest) 0.1 / dt, no accumulation and no clamp
  bool legacy = false;
  float bias = 0.0f, inv_sum = 0.0f;
  // a joint with no velocity row (a spring, or every row skipped) still solves at position level:
  // its one carrier row puts it in the schedule (a task of the reference's joint batches, which
  // hold every active joint, solver.rs:666-679) and does nothing in the velocity solve
  bool carrier = false;
};

// d6_hinge_axis (bodies.rs:891-901) at the restated feature set: -1 for none.
int d6_hinge_axis(const Joint& j);
// d6_row_angle (bodies.rs:908-918)
float d6_row_angle(const Joint& j, Q4 rot_a, Q4 rot_b, int i);
// d6_rows (solver.rs:336-424): the joint's velocity rows, appended to out.
void d6_rows(const World& w, const Joint& j, uint32_t joint, float dt, std::vector<JRow>& out);
// A joint's velocity rows whatever its kind (solver.rs:655-661): d6_rows, distance_rows
// (solver.rs:309-330) for an anchored distance joint, the original row for the others.
void joint_rows(const World& w, const Joint& j, uint32_t joint, float dt, std::vector<JRow>& out);
// joint_row_vel / joint_row_apply (solver.rs:291-307)
float joint_row_vel(const World& w, const JRow& r);
void joint_row_apply(World& w, const JRow& r, float lam);
// position_damped (bodies.rs:58-61)
bool position_damped(const D6Axis& a);
// One Gauss-Seidel update of a joint row (solver.rs:821-830); returns new - old.
float joint_row_update(World& w, const JRow& r, float& acc);
// Joints::solve_step_with for one sweep (bodies.rs:422-471) with SHAKE directions from start
// (indexed by body) and joints between two frozen bodies skipped.
void solve_joints_pass(World& w, float dt, const std::vector<Iso>& start, const std::vector<uint8_t>& frozen);

}  // namespace orc
