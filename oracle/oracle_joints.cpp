// oracle/oracle_joints.cpp -- TEST INFRASTRUCTURE (the oracle): D6 joints (ball, hinge, per-axis
// limits), their velocity rows and their XPBD position solve, restated from
// riftphys-articulation/src/bodies.rs and riftphys-world/src/world/solver.rs at the feature set
// the joint workloads use. Every fin / normalize of the reference is kept in place: those
// sanitations change bits. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
// reach this code.
#include "oracle_joints.h"

#include <cmath>

namespace orc {
using namespace om;

static const V3 kUnit[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
static const float kShakeMaxTurn = 0.5f;  // SHAKE_MAX_TURN (bodies.rs:477)
// SHAKE_MAX_TURN.cos() (bodies.rs:520), through the project's cosine
static float shake_max_turn_cos() {
  float s, c;
  om::sincosf_rp(kShakeMaxTurn, &s, &c);
  return c;
}
static const float kShakeMaxTurnCos = shake_max_turn_cos();

static inline float comp(V3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
// normalize_fin (bodies.rs:19-27)
static V3 normalize_fin(V3 v) {
  v = fin_v(v);
  float l2 = len2(v);
  if (l2 > 1.0e-12f) return mul(v, 1.0f / std::sqrt(l2));
  return V3{0, 0, 0};
}

// ---------------------------------------------------------------- joint construction
// Joints::add_ball (bodies.rs:326-331): translation locked, rotation free.
uint32_t World::add_ball_joint(uint32_t a, uint32_t b, const Iso& fa, const Iso& fb) {
  Joint j;
  j.a = a; j.b = b; j.fa = fa; j.fb = fb;
  for (int k = 0; k < 3; ++k) { j.t[k].enabled = true; j.r[k].enabled = false; }
  j.hinge = -1;
  joints.push_back(j);
  return (uint32_t)joints.size() - 1;
}
// Joints::add_hinge (bodies.rs:333-338): translation and the two other rotations locked.
uint32_t World::add_hinge_joint(uint32_t a, uint32_t b, const Iso& fa, const Iso& fb, uint32_t axis) {
  Joint j;
  j.a = a; j.b = b; j.fa = fa; j.fb = fb;
  for (int k = 0; k < 3; ++k) { j.t[k].enabled = true; j.r[k].enabled = (uint32_t)k != axis; }
  j.hinge = (int)axis;
  joints.push_back(j);
  return (uint32_t)joints.size() - 1;
}
// Joints::set_d6_limit_t / set_d6_limit_r (bodies.rs:367-372, 386-391) + leave_hinge (:876-878)
void World::set_d6_limit(uint32_t id, bool angular, uint32_t axis, bool has, float lo, float hi) {
  if (id >= joints.size() || axis > 2) return;
  Joint& j = joints[id];
  D6Axis& x = angular ? j.r[axis] : j.t[axis];
  x.has_limit = has;
  x.lo = lo; x.hi = hi;
  if (has) {
    x.enabled = true;
    if (angular && j.hinge >= 0 && j.hinge != (int)axis) j.hinge = -1;
  }
}
uint32_t World::add_d6_joint(uint32_t a, uint32_t b, const Iso& fa, const Iso& fb) {
  Joint j;
  j.a = a; j.b = b; j.fa = fa; j.fb = fb;
  for (int k = 0; k < 3; ++k) { j.t[k].enabled = true; j.r[k].enabled = true; }
  j.hinge = -1;
  joints.push_back(j);
  return (uint32_t)joints.size() - 1;
}
void World::set_d6_axis(uint32_t id, bool angular, uint32_t axis, bool enabled, float compliance) {
  if (id >= joints.size() || axis > 2) return;
  D6Axis& x = angular ? joints[id].r[axis] : joints[id].t[axis];
  x.enabled = enabled;
  x.compliance = compliance;
}
// Joints::set_d6_drive_t / set_d6_drive_r (bodies.rs:354-366)
void World::set_d6_drive(uint32_t id, bool angular, uint32_t axis, bool has, float target, float kp, float kd,
                         float max_impulse, bool vel_mode) {
  if (id >= joints.size() || axis > 2) return;
  Joint& j = joints[id];
  D6Axis& x = angular ? j.r[axis] : j.t[axis];
  x.has_drive = has;
  x.d_target = target; x.d_kp = kp; x.d_kd = kd; x.d_max = max_impulse; x.vel_mode = vel_mode;
  if (has) {
    x.enabled = true;
    if (angular && j.hinge >= 0 && j.hinge != (int)axis) j.hinge = -1;
  }
}
// Joints::set_d6_damping (bodies.rs:376-383): negative or non-finite values become 0
void World::set_d6_damping(uint32_t id, bool angular, uint32_t axis, float damping, float friction) {
  if (id >= joints.size() || axis > 2) return;
  D6Axis& x = angular ? joints[id].r[axis] : joints[id].t[axis];
  x.damping = rmax(fin0(damping), 0.0f);
  x.friction = rmax(fin0(friction), 0.0f);
}

// Joints::add_distance_joint (bodies.rs:273-285): rest and compliance sanitised (fin; compliance >= 0)
uint32_t World::add_distance_joint(uint32_t a, uint32_t b, float rest, float compliance) {
  Joint j;
  j.a = a; j.b = b; j.kind = 1;
  j.rest = fin0(rest);
  j.compliance = rmax(fin0(compliance), 0.0f);
  joints.push_back(j);
  return (uint32_t)joints.size() - 1;
}
// Joints::add_distance_joint_at (bodies.rs:290-297)
uint32_t World::add_distance_joint_at(uint32_t a, V3 la, uint32_t b, V3 lb, float rest, float compliance) {
  uint32_t id = add_distance_joint(a, b, rest, compliance);
  joints[id].la = fin_v(la);
  joints[id].lb = fin_v(lb);
  return id;
}
// Joints::set_distance_damping (bodies.rs:301-305)
void World::set_distance_damping(uint32_t id, float damping) {
  if (id >= joints.size() || joints[id].kind != 1) return;
  joints[id].damping = rmax(fin0(damping), 0.0f);
}

bool position_damped(const D6Axis& a) {
  return a.enabled && a.compliance > 0.0f && a.damping > 0.0f && !a.has_limit && (!a.has_drive || !a.vel_mode);
}

int d6_hinge_axis(const Joint& j) {
  if (j.hinge >= 0) return j.hinge < 3 ? j.hinge : -1;
  int free_axis = -1, n = 0;
  for (int i = 0; i < 3; ++i)
    if (!(j.r[i].enabled && !j.r[i].has_limit && !j.r[i].has_drive)) { free_axis = i; n++; }
  if (n == 1) return free_axis;
  auto c = [&](int i) { return j.r[i].enabled ? rmax(fin0(j.r[i].compliance), 0.0f) : 0.0f; };
  for (int i = 0; i < 3; ++i) {
    if (!(j.r[i].enabled && c(i) > 0.0f)) continue;
    bool all = true;
    for (int k = 0; k < 3; ++k) all = all && (k == i || c(i) >= 100.0f * c(k));
    if (all) return i;
  }
  return -1;
}

float d6_row_angle(const Joint& j, Q4 rot_a, Q4 rot_b, int i) {
  Q4 q = qmul(qconj(rot_a), rot_b);
  if (q.w < 0.0f) q = qneg(q);
  V3 v{q.x, q.y, q.z};
  if (d6_hinge_axis(j) == i) return 2.0f * atan2f_rp(comp(v, i), q.w);
  return dot(qrot(rot_a, mul(v, 2.0f)), qrot(rot_a, kUnit[i]));
}

// ---------------------------------------------------------------- velocity rows
void d6_rows(const World& w, const Joint& j, uint32_t joint, float dt, std::vector<JRow>& out) {
  const uint32_t a = j.a, b = j.b;
  Iso pa{w.pos[a], w.rot[a]}, pb{w.pos[b], w.rot[b]};
  Q4 rot_a = qmul(pa.rot, j.fa.rot), rot_b = qmul(pb.rot, j.fb.rot);
  V3 xa = add(pa.pos, qrot(pa.rot, j.fa.pos)), xb = add(pb.pos, qrot(pb.rot, j.fb.pos));
  V3 axes[3] = {qrot(rot_a, kUnit[0]), qrot(rot_a, kUnit[1]), qrot(rot_a, kUnit[2])};
  float wa = w.inv_mass[a], wb = w.inv_mass[b];
  if (wa == 0.0f && wb == 0.0f) return;
  M3 ia = w.inv_inertia_world(a), ib = w.inv_inertia_world(b);
  V3 ra = sub(xa, pa.pos), rb = sub(xb, pb.pos);
  V3 d = sub(xb, xa);
  for (int ang = 0; ang < 2; ++ang) {
    for (int i = 0; i < 3; ++i) {
      const D6Axis& row = ang ? j.r[i] : j.t[i];
      V3 u = axes[i];
      uint8_t tag = (uint8_t)((ang << 5) | (i << 3));
      auto keff = [&](V3 uu) {
        if (ang) return dot(uu, mvec(ia, uu)) + dot(uu, mvec(ib, uu));
        V3 ca = cross(ra, uu), cb = cross(rb, uu);
        return ((wa + wb) + dot(ca, mvec(ia, ca))) + dot(cb, mvec(ib, cb));
      };
      // joint damping and Coulomb friction (W3a), on any axis; a compliant damped row's damping
      // is in its position row instead
      float damp = position_damped(row) ? 0.0f : row.damping;
      if (damp > 0.0f || row.friction > 0.0f) {
        float kk = keff(u);
        if (kk > 1.0e-9f) {
          JRow base{a, b, joint, ang != 0, u, ra, rb, wa, wb, 1.0f / kk, 0.0f, -INFINITY, INFINITY, tag};
          if (damp > 0.0f) {
            JRow dr = base;
            dr.gamma = 1.0f / (damp * dt);
            dr.m_eff = 1.0f / (kk + dr.gamma);
            dr.tag = (uint8_t)(tag | 4);
            out.push_back(dr);
          }
          if (row.friction > 0.0f) {
            JRow fr = base;
            float cap = row.friction * dt;
            fr.lam_min = -cap; fr.lam_max = cap;
            fr.tag = (uint8_t)(tag | 5);
            out.push_back(fr);
          }
        }
      }
      if (!row.enabled || row.compliance > 0.0f) continue;
      if (row.has_drive && !row.vel_mode) continue;  // position drives stay at position level
      float k = keff(u);
      if (k <= 1.0e-9f) continue;
      JRow base{a, b, joint, ang != 0, u, ra, rb, wa, wb, 1.0f / k, 0.0f, -INFINITY, INFINITY, tag};
      if (row.has_drive) {  // velocity motor: the relative velocity to the target, at most max_impulse
        JRow mr = base;
        float cap = std::fabs(row.d_max);
        mr.target = row.d_target; mr.lam_min = -cap; mr.lam_max = cap;
        mr.tag = (uint8_t)(tag | 1);
        out.push_back(mr);
      }
      if (!row.has_limit) {
        if (!row.has_drive) out.push_back(base);
        continue;
      }
      float x = ang ? d6_row_angle(j, rot_a, rot_b, i) : dot(d, u);
      JRow lo = base, hi = base;
      lo.target = rmin((row.lo - x) / dt, 0.0f); lo.lam_min = 0.0f; lo.tag = (uint8_t)(tag | 2);
      hi.target = rmax((row.hi - x) / dt, 0.0f); hi.lam_max = 0.0f; hi.lam_min = -INFINITY; hi.tag = (uint8_t)(tag | 3);
      out.push_back(lo);
      out.push_back(hi);
    }
  }
}

// distance_rows (solver.rs:309-330): an anchored rigid rod's equality row along the current
// anchors' direction (a compliant rod has none: its damping is in its position row).
static void distance_rows(const World& w, const Joint& j, uint32_t joint, std::vector<JRow>& out) {
  const uint32_t a = j.a, b = j.b;
  float wa = w.inv_mass[a], wb = w.inv_mass[b];
  if (wa == 0.0f && wb == 0.0f) return;
  V3 ra = qrot(w.rot[a], j.la), rb = qrot(w.rot[b], j.lb);
  V3 d = sub(add(w.pos[b], rb), add(w.pos[a], ra));
  float len = om::len(d);
  if (!(len > 1e-6f)) return;
  V3 u = divs(d, len);
  M3 ia = w.inv_inertia_world(a), ib = w.inv_inertia_world(b);
  V3 ca = cross(ra, u), cb = cross(rb, u);
  float k = ((wa + wb) + dot(ca, mvec(ia, ca))) + dot(cb, mvec(ib, cb));
  if (!(k > 1e-9f)) return;
  if (j.compliance <= 0.0f) out.push_back(JRow{a, b, joint, false, u, ra, rb, wa, wb, 1.0f / k, 0.0f, -INFINITY, INFINITY, 0});
}
// The original distance row (solver.rs:793-817), made once per tick: positions do not move
// during the velocity solve, so its direction and bias are the same at every sweep.
static void legacy_distance_row(const World& w, const Joint& j, uint32_t joint, float dt, std::vector<JRow>& out) {
  if (j.compliance > 0.0f) return;  // a spring acts at position level only
  V3 dir = sub(w.pos[j.b], w.pos[j.a]);
  float len = om::len(dir);
  if (len < 1e-6f) return;
  V3 n = divs(dir, len);
  float inv_a = w.inv_mass[j.a], inv_b = w.inv_mass[j.b];
  float inv_sum = inv_a + inv_b;
  if (inv_sum < 1e-9f) return;
  JRow r{j.a, j.b, joint, false, n, V3{0, 0, 0}, V3{0, 0, 0}, inv_a, inv_b, 1.0f / inv_sum, 0.0f, -INFINITY, INFINITY, 0};
  r.legacy = true;
  r.bias = (len - j.rest) * (0.1f / dt);
  r.inv_sum = inv_sum;
  out.push_back(r);
}
void joint_rows(const World& w, const Joint& j, uint32_t joint, float dt, std::vector<JRow>& out) {
  const size_t s0 = out.size();
  if (j.kind == 0) d6_rows(w, j, joint, dt, out);
  else if (j.anchored()) distance_rows(w, j, joint, out);
  else legacy_distance_row(w, j, joint, dt, out);
  float wa = w.inv_mass[j.a], wb = w.inv_mass[j.b];
  if (out.size() == s0 && (wa > 0.0f || wb > 0.0f)) {
    JRow r{j.a, j.b, joint, false, V3{0, 0, 0}, V3{0, 0, 0}, V3{0, 0, 0}, wa, wb, 1.0f, 0.0f, -INFINITY, INFINITY, 0};
    r.carrier = true;
    out.push_back(r);
  }
}

float joint_row_vel(const World& w, const JRow& r) {
  if (r.angular) return dot(sub(w.ang[r.b], w.ang[r.a]), r.u);
  V3 vb = add(w.lin[r.b], cross(w.ang[r.b], r.rb));
  V3 va = add(w.lin[r.a], cross(w.ang[r.a], r.ra));
  return dot(sub(vb, va), r.u);
}
void joint_row_apply(World& w, const JRow& r, float lam) {
  V3 p = mul(r.u, lam);
  if (r.angular) {
    if (r.wa > 0.0f) w.apply_angular_impulse(r.a, neg(p));
    if (r.wb > 0.0f) w.apply_angular_impulse(r.b, p);
  } else {
    if (r.wa > 0.0f) { w.apply_impulse(r.a, neg(p)); w.apply_angular_impulse(r.a, cross(r.ra, neg(p))); }
    if (r.wb > 0.0f) { w.apply_impulse(r.b, p); w.apply_angular_impulse(r.b, cross(r.rb, p)); }
  }
}
float joint_row_update(World& w, const JRow& r, float& acc) {
  if (r.carrier) return 0.0f;
  if (r.legacy) {
    float v_rel = dot(sub(w.lin[r.b], w.lin[r.a]), r.u);
    float j_mag = -(v_rel + r.bias) / r.inv_sum;
    w.apply_impulse(r.a, mul(neg(r.u), j_mag));
    w.apply_impulse(r.b, mul(r.u, j_mag));
    return j_mag;
  }
  float v = joint_row_vel(w, r);
  float old = acc;
  // rigid rows: v -> target; soft rows (dampers): v + gamma lam -> target
  float nw = r.gamma == 0.0f ? old + (r.target - v) * r.m_eff : old + ((r.target - v) - r.gamma * old) * r.m_eff;
  nw = clampf(nw, r.lam_min, r.lam_max);
  acc = nw;
  if (nw != old) joint_row_apply(w, r, nw - old);
  return nw - old;
}

// ---------------------------------------------------------------- position solve
// Bodies::apply_position_delta / apply_orientation_delta (dynamics.rs:71-88, 207-210)
static void apply_position_delta(World& w, uint32_t id, V3 dp) {
  if (w.inv_mass[id] > 0.0f && vfin(dp)) w.pos[id] = fin_v(add(w.pos[id], dp));
}
static Q4 fin_q(Q4 q) {
  if (!qfin(q)) return Q4{0, 0, 0, 1};
  Q4 qq = qnormalize(q);
  if (!qfin(qq)) return Q4{0, 0, 0, 1};
  if (qq.w < 0.0f) qq = qneg(qq);
  return qq;
}
static void apply_orientation_delta(World& w, uint32_t id, V3 dth) {
  if (w.inv_mass[id] <= 0.0f || !vfin(dth)) return;
  V3 d = fin_v(dth);
  if (len2(d) <= 1.0e-24f) return;
  Q4 dq = qnormalize(Q4{d.x * 0.5f, d.y * 0.5f, d.z * 0.5f, 1.0f});
  w.rot[id] = fin_q(qnormalize(qmul(dq, w.rot[id])));
}
// turned (bodies.rs:486-490): rotation between two orientations, radians
static float turned(Q4 a, Q4 b) {
  float d = rmin(std::fabs(qmul(a, qconj(b)).w), 1.0f);
  return 2.0f * acosf_unit_rp(d);
}
// inv_inertia_at (bodies.rs:493-497)
static M3 inv_inertia_at(const World& w, uint32_t id, Q4 rot) {
  M3 r = mfrom_quat(rot);
  return mmul(mmul(r, w.inv_I[id]), mtranspose(r));
}
// alpha_dt2 (bodies.rs:438-441)
static float alpha_dt2(float c, float dt2) {
  c = rmax(fin0(c), 0.0f);
  return c <= 0.0f ? 0.0f : fin0(c / dt2);
}
// The error a row acts on (bodies.rs:674-698, 786-810): locked at 0, a limit only while violated,
// a position drive's target (clamped into the limit); a velocity drive leaves the axis free at
// position level unless it is limited. False: nothing to correct.
static bool row_error(const D6Axis& row, float coord, float* c) {
  bool has = true;
  *c = fin0(coord - 0.0f);
  if (row.has_limit) {
    float lo = fin0(row.lo), hi = fin0(row.hi);
    if (coord < lo) *c = fin0(coord - lo);
    else if (coord > hi) *c = fin0(coord - hi);
    else has = false;
  }
  if (row.has_drive) {
    if (!row.vel_mode) {
      float target = fin0(row.d_target);
      if (row.has_limit) target = clampf(target, fin0(row.lo), fin0(row.hi));
      *c = fin0(coord - target);
      has = true;
    } else if (!row.has_limit) {
      has = false;
    }
  }
  return has;
}
// The measure of rotational row i at joint-frame rotations ra, rb (bodies.rs:796-803).
static float row_angle(int hinge, Q4 ra, Q4 rb, int i, V3 u) {
  Q4 q = qmul(qconj(ra), rb);
  if (q.w < 0.0f) q = qneg(q);
  V3 v{q.x, q.y, q.z};
  if (hinge == i) return fin0(2.0f * atan2f_rp(comp(v, i), q.w));
  if (hinge >= 0)
    return fin0(dot(fin_v(cross(normalize_fin(qrot(ra, kUnit[hinge])), normalize_fin(qrot(rb, kUnit[hinge])))), u));
  return fin0(dot(fin_v(qrot(ra, fin_v(mul(v, 2.0f)))), u));
}

// solve_d6 (bodies.rs:616-873) without the rotor rows (no armature). sa / sb: the step's start
// poses, for SHAKE's directions (when neither body turned too far) and for a damped compliant
// row's change since the start.
static void solve_d6(World& w, Joint& j, float dt, const Iso* sa, const Iso* sb) {
  const float wa = fin0(w.inv_mass[j.a]), wb = fin0(w.inv_mass[j.b]);
  const float dt2 = rmax(dt * dt, 1.0e-12f);
  Q4 ra0_rot = w.rot[j.a], rb0_rot = w.rot[j.b];
  bool shake = sa && sb && turned(sa->rot, ra0_rot) < kShakeMaxTurn && turned(sb->rot, rb0_rot) < kShakeMaxTurn;
  V3 ax0[3] = {}, la0{}, lb0{};
  M3 ia0 = mzero(), ib0 = mzero();
  if (shake) {
    Q4 r0 = qmul(sa->rot, j.fa.rot);
    for (int i = 0; i < 3; ++i) ax0[i] = normalize_fin(qrot(r0, kUnit[i]));
    la0 = fin_v(qrot(sa->rot, j.fa.pos));
    lb0 = fin_v(qrot(sb->rot, j.fb.pos));
    ia0 = inv_inertia_at(w, j.a, sa->rot);
    ib0 = inv_inertia_at(w, j.b, sb->rot);
  }
  const float bias_vel = 0.0f;
  for (int i = 0; i < 3; ++i) {
    const D6Axis& row = j.t[i];
    if (!row.enabled) continue;
    Iso pa{w.pos[j.a], w.rot[j.a]}, pb{w.pos[j.b], w.rot[j.b]};
    V3 u = normalize_fin(qrot(qmul(pa.rot, j.fa.rot), kUnit[i]));
    if (vzero(u)) continue;
    V3 xa = fin_v(add(pa.pos, qrot(pa.rot, j.fa.pos)));
    V3 xb = fin_v(add(pb.pos, qrot(pb.rot, j.fb.pos)));
    V3 d = fin_v(sub(xb, xa));
    V3 un, lever_a, lever_b;
    M3 iaw, ibw;
    if (shake) { un = ax0[i]; lever_a = la0; lever_b = lb0; iaw = ia0; ibw = ib0; }
    else {
      un = u; lever_a = sub(xa, pa.pos); lever_b = sub(xb, pb.pos);
      iaw = w.inv_inertia_world(j.a); ibw = w.inv_inertia_world(j.b);
    }
    float coord = fin0(dot(d, u));
    float c;
    if (!row_error(row, coord, &c)) continue;
    V3 ra_u = fin_v(cross(lever_a, un)), rb_u = fin_v(cross(lever_b, un));
    float w_rot_a = fin0(dot(ra_u, mvec(iaw, ra_u)));
    float w_rot_b = fin0(dot(rb_u, mvec(ibw, rb_u)));
    float ws = fin0(((wa + wb) + w_rot_a) + w_rot_b);
    float alpha = alpha_dt2(row.compliance, dt2);
    float denom = fin0(ws + alpha);
    if (denom <= 0.0f) continue;
    c = fin0(c + fin0(bias_vel * dt));
    float lambda_old = fin0(j.lam_t[i]);
    float dl;
    if (position_damped(row) && sa && sb) {  // Kelvin-Voigt: spring and damper in one implicit row
      V3 u0 = normalize_fin(qrot(qmul(sa->rot, j.fa.rot), kUnit[i]));
      V3 d0 = fin_v(sub(add(sb->pos, qrot(sb->rot, j.fb.pos)), add(sa->pos, qrot(sa->rot, j.fa.pos))));
      float gamma = fin0(row.compliance * row.damping / dt);
      float dc = fin0(coord - dot(d0, u0));
      dl = fin0(-((c + fin0(alpha * lambda_old)) + fin0(gamma * dc)) / fin0((1.0f + gamma) * ws + alpha));
    } else {
      dl = fin0(-(c + fin0(alpha * lambda_old)) / denom);
    }
    j.lam_t[i] = fin0(lambda_old + dl);
    apply_position_delta(w, j.a, fin_v(mul(neg(un), fin0(dl * wa))));
    apply_position_delta(w, j.b, fin_v(mul(un, fin0(dl * wb))));
    apply_orientation_delta(w, j.a, fin_v(mul(neg(mvec(iaw, ra_u)), dl)));
    apply_orientation_delta(w, j.b, fin_v(mul(mvec(ibw, rb_u), dl)));
  }
  const int hinge = d6_hinge_axis(j);
  for (int i = 0; i < 3; ++i) {
    const D6Axis& row = j.r[i];
    if (!row.enabled) continue;
    Q4 ra = qmul(w.rot[j.a], j.fa.rot), rb = qmul(w.rot[j.b], j.fb.rot);
    V3 u = normalize_fin(qrot(ra, kUnit[i]));
    if (vzero(u)) continue;
    float angle = row_angle(hinge, ra, rb, i, u);
    V3 un;
    M3 iaw, ibw;
    if (shake) { un = ax0[i]; iaw = ia0; ibw = ib0; }
    else { un = u; iaw = w.inv_inertia_world(j.a); ibw = w.inv_inertia_world(j.b); }
    float c;
    if (!row_error(row, angle, &c)) continue;
    float ws = fin0(dot(un, mvec(iaw, un)) + dot(un, mvec(ibw, un)));
    float alpha = alpha_dt2(row.compliance, dt2);
    float denom = fin0(ws + alpha);
    if (denom <= 0.0f) continue;
    c = fin0(c + fin0(bias_vel * dt));
    float lambda_old = fin0(j.lam_r[i]);
    float dl;
    if (position_damped(row) && sa && sb) {
      Q4 ra0 = qmul(sa->rot, j.fa.rot), rb0 = qmul(sb->rot, j.fb.rot);
      V3 u0 = normalize_fin(qrot(ra0, kUnit[i]));
      float angle0 = row_angle(hinge, ra0, rb0, i, u0);
      float gamma = fin0(row.compliance * row.damping / dt);
      float dc = fin0(angle - angle0);
      dl = fin0(-((c + fin0(alpha * lambda_old)) + fin0(gamma * dc)) / fin0((1.0f + gamma) * ws + alpha));
    } else {
      dl = fin0(-(c + fin0(alpha * lambda_old)) / denom);
    }
    j.lam_r[i] = fin0(lambda_old + dl);
    apply_orientation_delta(w, j.a, fin_v(mul(neg(mvec(iaw, un)), dl)));
    apply_orientation_delta(w, j.b, fin_v(mul(mvec(ibw, un), dl)));
  }
}

// solve_distance_row (bodies.rs:501-548): the original COM-to-COM rod, corrected along the
// start-of-step direction when it is within SHAKE_MAX_TURN of the current one.
static void solve_distance_row(World& w, Joint& j, float dt2, const Iso* sa, const Iso* sb) {
  const uint32_t ia = j.a, ib = j.b;
  float wa = w.inv_mass[ia], wb = w.inv_mass[ib];
  float w_sum = fin0(wa + wb);
  if (w_sum <= 0.0f) return;
  V3 d = sub(w.pos[ib], w.pos[ia]);
  float len2 = dot(d, d);
  if (!fin(len2) || len2 <= 1.0e-20f) return;
  float len = std::sqrt(len2);
  if (len <= 1.0e-6f) return;
  V3 n_cur = normalize_fin(divs(d, len));
  if (vzero(n_cur)) return;
  V3 n = n_cur;
  if (sa && sb) {
    V3 n0 = normalize_fin(sub(sb->pos, sa->pos));
    if (!vzero(n0) && dot(n0, n_cur) > kShakeMaxTurnCos) n = n0;
  }
  float c_val = fin0(len - fin0(j.rest));
  float alpha = j.compliance <= 0.0f ? 0.0f : fin0(rmax(fin0(j.compliance), 0.0f) / dt2);
  float denom = fin0(w_sum + alpha);
  if (denom <= 0.0f) return;
  float lambda_old = fin0(j.lambda_acc);
  float lambda = fin0(-(c_val + fin0(alpha * lambda_old)) / (denom * dot(n, n_cur)));
  if (std::fabs(lambda) <= 1.0e-9f) return;
  j.lambda_acc = fin0(lambda_old + lambda);
  apply_position_delta(w, ia, fin_v(mul(neg(n), fin0(lambda * wa))));
  apply_position_delta(w, ib, fin_v(mul(n, fin0(lambda * wb))));
}
// solve_distance_anchored (bodies.rs:557-614): C = |x_b - x_a| - rest on the current anchors,
// along the start-of-step direction with start-of-step lever arms and inertias over the mixed
// Jacobian product (current-iterate directions when a body turned too far or the mixed product
// falls below half the start-of-step one); a damped compliant rod's spring and damper in one
// implicit Kelvin-Voigt row.
static void solve_distance_anchored(World& w, Joint& j, float dt, float dt2, const Iso* sa, const Iso* sb) {
  const uint32_t ia = j.a, ib = j.b;
  float wa = fin0(w.inv_mass[ia]), wb = fin0(w.inv_mass[ib]);
  if (wa + wb <= 0.0f) return;
  Iso pa{w.pos[ia], w.rot[ia]}, pb{w.pos[ib], w.rot[ib]};
  V3 ra = fin_v(qrot(pa.rot, j.la)), rb = fin_v(qrot(pb.rot, j.lb));
  V3 d = fin_v(sub(add(pb.pos, rb), add(pa.pos, ra)));
  float len = om::len(d);
  if (!fin(len) || len <= 1.0e-6f) return;
  V3 n_cur = normalize_fin(divs(d, len));
  if (vzero(n_cur)) return;
  float c_val = fin0(len - fin0(j.rest));
  float alpha = j.compliance <= 0.0f ? 0.0f : fin0(rmax(fin0(j.compliance), 0.0f) / dt2);
  V3 n, ga, gb;
  float wgen;
  bool shake = false;
  if (sa && sb && !(turned(sa->rot, pa.rot) >= kShakeMaxTurn) && !(turned(sb->rot, pb.rot) >= kShakeMaxTurn)) {
    V3 ra0 = qrot(sa->rot, j.la), rb0 = qrot(sb->rot, j.lb);
    V3 n0 = normalize_fin(sub(add(sb->pos, rb0), add(sa->pos, ra0)));
    if (!vzero(n0)) {
      M3 ia0 = inv_inertia_at(w, ia, sa->rot), ib0 = inv_inertia_at(w, ib, sb->rot);
      V3 ga0 = mvec(ia0, cross(ra0, n0)), gb0 = mvec(ib0, cross(rb0, n0));
      float w_sym = ((wa + wb) + dot(cross(ra0, n0), ga0)) + dot(cross(rb0, n0), gb0);
      float w_mix = (((wa + wb) * dot(n_cur, n0)) + dot(cross(ra, n_cur), ga0)) + dot(cross(rb, n_cur), gb0);
      if (fin(w_mix) && w_mix >= 0.5f * w_sym) { shake = true; n = n0; ga = ga0; gb = gb0; wgen = w_mix; }
    }
  }
  if (!shake) {
    M3 iaw = w.inv_inertia_world(ia), ibw = w.inv_inertia_world(ib);
    V3 ca = cross(ra, n_cur), cb = cross(rb, n_cur);
    wgen = ((wa + wb) + dot(ca, mvec(iaw, ca))) + dot(cb, mvec(ibw, cb));
    n = n_cur; ga = mvec(iaw, ca); gb = mvec(ibw, cb);
  }
  float denom = fin0(wgen + alpha);
  if (!(denom > 0.0f)) return;
  float lambda_old = fin0(j.lambda_acc);
  float dl;
  if (j.compliance > 0.0f && j.damping > 0.0f && sa && sb) {
    float len0 = om::len(sub(add(sb->pos, qrot(sb->rot, j.lb)), add(sa->pos, qrot(sa->rot, j.la))));
    float gamma = fin0(j.compliance * j.damping / dt);
    dl = fin0(-((c_val + fin0(alpha * lambda_old)) + fin0(gamma * fin0(len - len0))) / fin0((1.0f + gamma) * wgen + alpha));
  } else {
    dl = fin0(-(c_val + fin0(alpha * lambda_old)) / denom);
  }
  if (std::fabs(dl) <= 1.0e-12f) return;
  j.lambda_acc = fin0(lambda_old + dl);
  apply_position_delta(w, ia, fin_v(mul(neg(n), fin0(dl * wa))));
  apply_position_delta(w, ib, fin_v(mul(n, fin0(dl * wb))));
  apply_orientation_delta(w, ia, fin_v(mul(neg(ga), dl)));
  apply_orientation_delta(w, ib, fin_v(mul(gb, dl)));
}

void solve_joints_pass(World& w, float dt, const std::vector<Iso>& start, const std::vector<uint8_t>& frozen) {
  dt = fin0(dt);
  if (!(dt > 0.0f)) return;
  for (auto& j : w.joints) {
    bool fa = j.a < frozen.size() ? frozen[j.a] != 0 : false;
    bool fb = j.b < frozen.size() ? frozen[j.b] != 0 : false;
    if (fa && fb) continue;
    const Iso* sa = j.a < start.size() ? &start[j.a] : nullptr;
    const Iso* sb = j.b < start.size() ? &start[j.b] : nullptr;
    Iso ca{w.pos[j.a], w.rot[j.a]}, cb{w.pos[j.b], w.rot[j.b]};
    if (j.kind == 0) solve_d6(w, j, dt, sa ? sa : &ca, sb ? sb : &cb);
    else if (j.anchored()) solve_distance_anchored(w, j, dt, rmax(dt * dt, 1.0e-12f), sa ? sa : &ca, sb ? sb : &cb);
    else solve_distance_row(w, j, rmax(dt * dt, 1.0e-12f), sa ? sa : &ca, sb ? sb : &cb);
  }
}

}  // namespace orc
