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

int d6_hinge_axis(const Joint& j) {
  if (j.hinge >= 0) return j.hinge < 3 ? j.hinge : -1;
  int free_axis = -1, n = 0;
  for (int i = 0; i < 3; ++i)
    if (!(j.r[i].enabled && !j.r[i].has_limit)) { free_axis = i; n++; }
  if (n == 1) return free_axis;
  return -1;  // the compliance rule needs a compliant row; none is restated
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
      if (!row.enabled) continue;
      float k;
      if (ang) k = dot(u, mvec(ia, u)) + dot(u, mvec(ib, u));
      else {
        V3 ca = cross(ra, u), cb = cross(rb, u);
        k = ((wa + wb) + dot(ca, mvec(ia, ca))) + dot(cb, mvec(ib, cb));
      }
      if (k <= 1.0e-9f) continue;
      JRow base{a, b, joint, ang != 0, u, ra, rb, wa, wb, 1.0f / k, 0.0f, -INFINITY, INFINITY, tag};
      if (!row.has_limit) { out.push_back(base); continue; }
      float x = ang ? d6_row_angle(j, rot_a, rot_b, i) : dot(d, u);
      JRow lo = base, hi = base;
      lo.target = rmin((row.lo - x) / dt, 0.0f); lo.lam_min = 0.0f; lo.tag = (uint8_t)(tag | 2);
      hi.target = rmax((row.hi - x) / dt, 0.0f); hi.lam_max = 0.0f; hi.lam_min = -INFINITY; hi.tag = (uint8_t)(tag | 3);
      out.push_back(lo);
      out.push_back(hi);
    }
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
  float v = joint_row_vel(w, r);
  float old = acc;
  float nw = clampf(old + (r.target - v) * r.m_eff, r.lam_min, r.lam_max);
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

// solve_d6 (bodies.rs:616-873) for locked and limited axes (no drive, compliance 0, so alpha = 0
// and every row is the plain XPBD step).
static void solve_d6(World& w, Joint& j, float dt, const Iso* sa, const Iso* sb) {
  const float wa = fin0(w.inv_mass[j.a]), wb = fin0(w.inv_mass[j.b]);
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
  const float alpha = 0.0f, bias_vel = 0.0f;
  auto limit_err = [](const D6Axis& row, float coord, float* c) {
    *c = fin0(coord - 0.0f);
    if (!row.has_limit) return true;
    float lo = fin0(row.lo), hi = fin0(row.hi);
    if (coord < lo) { *c = fin0(coord - lo); return true; }
    if (coord > hi) { *c = fin0(coord - hi); return true; }
    return false;
  };
  for (int i = 0; i < 3; ++i) {
    if (!j.t[i].enabled) continue;
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
    if (!limit_err(j.t[i], coord, &c)) continue;
    V3 ra_u = fin_v(cross(lever_a, un)), rb_u = fin_v(cross(lever_b, un));
    float w_rot_a = fin0(dot(ra_u, mvec(iaw, ra_u)));
    float w_rot_b = fin0(dot(rb_u, mvec(ibw, rb_u)));
    float ws = fin0(((wa + wb) + w_rot_a) + w_rot_b);
    float denom = fin0(ws + alpha);
    if (denom <= 0.0f) continue;
    c = fin0(c + fin0(bias_vel * dt));
    float lambda_old = fin0(j.lam_t[i]);
    float dl = fin0(-(c + fin0(alpha * lambda_old)) / denom);
    j.lam_t[i] = fin0(lambda_old + dl);
    apply_position_delta(w, j.a, fin_v(mul(neg(un), fin0(dl * wa))));
    apply_position_delta(w, j.b, fin_v(mul(un, fin0(dl * wb))));
    apply_orientation_delta(w, j.a, fin_v(mul(neg(mvec(iaw, ra_u)), dl)));
    apply_orientation_delta(w, j.b, fin_v(mul(mvec(ibw, rb_u), dl)));
  }
  const int hinge = d6_hinge_axis(j);
  for (int i = 0; i < 3; ++i) {
    if (!j.r[i].enabled) continue;
    Q4 ra = qmul(w.rot[j.a], j.fa.rot), rb = qmul(w.rot[j.b], j.fb.rot);
    V3 u = normalize_fin(qrot(ra, kUnit[i]));
    if (vzero(u)) continue;
    Q4 q = qmul(qconj(ra), rb);
    if (q.w < 0.0f) q = qneg(q);
    V3 v{q.x, q.y, q.z};
    float angle;
    if (hinge == i) angle = fin0(2.0f * atan2f_rp(comp(v, i), q.w));
    else if (hinge >= 0)
      angle = fin0(dot(fin_v(cross(normalize_fin(qrot(ra, kUnit[hinge])), normalize_fin(qrot(rb, kUnit[hinge])))), u));
    else angle = fin0(dot(fin_v(qrot(ra, fin_v(mul(v, 2.0f)))), u));
    V3 un;
    M3 iaw, ibw;
    if (shake) { un = ax0[i]; iaw = ia0; ibw = ib0; }
    else { un = u; iaw = w.inv_inertia_world(j.a); ibw = w.inv_inertia_world(j.b); }
    float c;
    if (!limit_err(j.r[i], angle, &c)) continue;
    float ws = fin0(dot(un, mvec(iaw, un)) + dot(un, mvec(ibw, un)));
    float denom = fin0(ws + alpha);
    if (denom <= 0.0f) continue;
    c = fin0(c + fin0(bias_vel * dt));
    float lambda_old = fin0(j.lam_r[i]);
    float dl = fin0(-(c + fin0(alpha * lambda_old)) / denom);
    j.lam_r[i] = fin0(lambda_old + dl);
    apply_orientation_delta(w, j.a, fin_v(mul(neg(mvec(iaw, un)), dl)));
    apply_orientation_delta(w, j.b, fin_v(mul(mvec(ibw, un), dl)));
  }
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
    solve_d6(w, j, dt, sa ? sa : &ca, sb ? sb : &cb);
  }
}

}  // namespace orc
