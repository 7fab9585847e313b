// joints.cuh -- D6 joints on the GPU: the joint record the kernels read, its velocity rows
// (d6_rows, riftphys-world/src/world/solver.rs:336-424) and its XPBD position solve with SHAKE
// directions (solve_d6, riftphys-articulation/src/bodies.rs:616-873): locked, limited, compliant
// and driven axes, joint damping and friction (no armature rotors).
// Every fin / normalize of the reference is kept where it stands: those sanitations change bits.
#pragma once
#include "step_rows.cuh"

namespace rp {

// One joint, 256 bytes. flags: bit i (i < 6) axis i enabled (t0 t1 t2 r0 r1 r2), bit 6 + i axis i
// limited to [lo[i], hi[i]], bits 12..14 the hinge axis + 1 (0: none; d6_hinge_axis, resolved on
// the host whenever the joint changes), bit 16 + i axis i driven, bit 22 + i that drive a velocity
// motor. Per axis: XPBD compliance, damping, friction, drive target and impulse cap.
struct JointGpu {
  uint32_t a, b, flags, pad;
  float4 fa_p, fa_q, fb_p, fb_q;
  float lo[6], hi[6];
  float comp[6], damp[6], fric[6], dtarget[6], dmax[6];
  float pad2[2];
};
static_assert(sizeof(JointGpu) == 256, "JointGpu layout");
#define JF_LIMIT_SHIFT 6u
#define JF_HINGE_SHIFT 12u
#define JF_DRIVE_SHIFT 16u
#define JF_VEL_SHIFT 22u
#define JF_FULL (1u << 28)  // some axis compliant or driven: the position solve takes the full path
// A distance joint (DistanceJoint, bodies.rs:31-51): rest length lo[0], compliance comp[0],
// damping damp[0], anchors fa_p.xyz / fb_p.xyz in each body's frame; JF_ANCH: anchored (an anchor
// or damping set), solved by the anchored rows, else by the original COM-to-COM ones.
#define JF_DIST (1u << 29)
#define JF_ANCH (1u << 30)
#define JMAX_ROWS kJointRows

__host__ __device__ inline int joint_hinge(uint32_t flags) { return (int)((flags >> JF_HINGE_SHIFT) & 7u) - 1; }

// A joint velocity row (JointRow, solver.rs:264-288); gamma = 1 / (damping dt) on a damper row.
// legacy: the original distance row (solver.rs:793-817), impulse -(v_rel + bias) / inv_sum along u
// on the linear velocities, no accumulation and no clamp.
struct JRowD {
  f3 u, ra, rb;
  float wa, wb, m_eff, target, lo, hi, gamma;
  uint32_t tag;
  bool angular;
  bool legacy = false;
  float bias = 0.0f, inv_sum = 0.0f;
  bool carrier = false;  // a joint's one row when it has no velocity row (RF_JNULL)
};
__host__ __device__ inline bool jaxis_on(uint32_t f, int ax) { return (f >> ax) & 1u; }
__host__ __device__ inline bool jaxis_lim(uint32_t f, int ax) { return (f >> (JF_LIMIT_SHIFT + ax)) & 1u; }
__host__ __device__ inline bool jaxis_drive(uint32_t f, int ax) { return (f >> (JF_DRIVE_SHIFT + ax)) & 1u; }
__host__ __device__ inline bool jaxis_vel(uint32_t f, int ax) { return (f >> (JF_VEL_SHIFT + ax)) & 1u; }
// position_damped (bodies.rs:58-61)
__device__ __forceinline__ bool position_damped_dev(const JointGpu& j, int ax) {
  return jaxis_on(j.flags, ax) && j.comp[ax] > 0.0f && j.damp[ax] > 0.0f && !jaxis_lim(j.flags, ax) &&
         (!jaxis_drive(j.flags, ax) || !jaxis_vel(j.flags, ax));
}

__device__ __forceinline__ f3 unit_axis(int i) { return i == 0 ? mk3(1, 0, 0) : (i == 1 ? mk3(0, 1, 0) : mk3(0, 0, 1)); }
__device__ __forceinline__ float comp3(f3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
// normalize_fin (bodies.rs:19-27)
__device__ __forceinline__ f3 normalize_fin(f3 v) {
  v = fin_v(v);
  float l2 = len2(v);
  if (l2 > 1.0e-12f) return v * (1.0f / sqrtf(l2));
  return mk3(0, 0, 0);
}
// d6_row_angle (bodies.rs:908-918)
__device__ __forceinline__ float d6_row_angle_dev(int hinge, q4 rot_a, q4 rot_b, int i) {
  q4 q = qmul(qconj(rot_a), rot_b);
  if (q.w < 0.0f) q = qneg(q);
  f3 v = mk3(q.x, q.y, q.z);
  if (hinge == i) return 2.0f * atan2_rp(comp3(v, i), q.w);
  return dot(qrot(rot_a, v * 2.0f), qrot(rot_a, unit_axis(i)));
}
// World inverse inertia the way Bodies::inv_inertia_world gives it (zero for inv_mass 0).
__device__ __forceinline__ m3 inv_inertia_world_dev(const BodiesV& B, uint32_t id, q4 rot) {
  if (B.inv_mass[id] == 0.0f) return mzero();
  return world_inertia(rot, ld_m3(B.inv_I, id));
}

// d6_rows (solver.rs:336-424): per axis, in (linear x y z, angular x y z) order, a damper row and a
// friction row when set (any axis; a compliant damped row's damping stays in its position row),
// then for an enabled rigid axis without a position drive a motor row (velocity drive) and either
// the equality row (no limit, no drive) or the two limit rows. Returns the row count (0 when
// neither body is dynamic). Each row goes to emit(row, index in the joint) as it is made.
template <class Emit>
__device__ __forceinline__ uint32_t d6_rows_dev(const JointGpu& j, const BodiesV& B, float dt, Emit&& emit) {
  const uint32_t a = j.a, b = j.b;
  f3 pa = xyz(B.pos[a]), pb = xyz(B.pos[b]);
  q4 qa = asq(B.rot[a]), qb = asq(B.rot[b]);
  q4 rot_a = qmul(qa, asq(j.fa_q)), rot_b = qmul(qb, asq(j.fb_q));
  f3 xa = pa + qrot(qa, xyz(j.fa_p)), xb = pb + qrot(qb, xyz(j.fb_p));
  float wa = B.inv_mass[a], wb = B.inv_mass[b];
  if (wa == 0.0f && wb == 0.0f) return 0;
  m3 ia = wa == 0.0f ? mzero() : ld_m3(B.Iw, a), ib = wb == 0.0f ? mzero() : ld_m3(B.Iw, b);
  f3 ra = xa - pa, rb = xb - pb, d = xb - xa;
  const int hinge = joint_hinge(j.flags);
  uint32_t n = 0;
  for (int ang = 0; ang < 2; ++ang) {
    for (int i = 0; i < 3; ++i) {
      const int ax = 3 * ang + i;
      f3 u = qrot(rot_a, unit_axis(i));
      auto keff = [&]() {
        if (ang) return dot(u, mvec(ia, u)) + dot(u, mvec(ib, u));
        f3 ca = cross(ra, u), cb = cross(rb, u);
        return ((wa + wb) + dot(ca, mvec(ia, ca))) + dot(cb, mvec(ib, cb));
      };
      JRowD base;
      base.u = u; base.ra = ra; base.rb = rb; base.wa = wa; base.wb = wb;
      base.target = 0.0f; base.lo = -INFINITY; base.hi = INFINITY; base.gamma = 0.0f;
      base.tag = (uint32_t)((ang << 5) | (i << 3));
      base.angular = ang != 0;
      const float damp = position_damped_dev(j, ax) ? 0.0f : j.damp[ax];
      if (damp > 0.0f || j.fric[ax] > 0.0f) {
        float kk = keff();
        if (kk > 1.0e-9f) {
          if (damp > 0.0f) {
            JRowD r = base;
            r.gamma = 1.0f / (damp * dt);
            r.m_eff = 1.0f / (kk + r.gamma);
            r.tag = base.tag | 4u;
            emit(r, n++);
          }
          if (j.fric[ax] > 0.0f) {
            JRowD r = base;
            r.m_eff = 1.0f / kk;
            float cap = j.fric[ax] * dt;
            r.lo = -cap; r.hi = cap;
            r.tag = base.tag | 5u;
            emit(r, n++);
          }
        }
      }
      if (!jaxis_on(j.flags, ax) || j.comp[ax] > 0.0f) continue;
      const bool drive = jaxis_drive(j.flags, ax), vel = jaxis_vel(j.flags, ax);
      if (drive && !vel) continue;  // position drives stay at position level
      float k = keff();
      if (k <= 1.0e-9f) continue;
      base.m_eff = 1.0f / k;
      if (drive) {  // velocity motor
        JRowD r = base;
        float cap = fabsf(j.dmax[ax]);
        r.target = j.dtarget[ax]; r.lo = -cap; r.hi = cap;
        r.tag = base.tag | 1u;
        emit(r, n++);
      }
      if (!jaxis_lim(j.flags, ax)) {
        if (!drive) emit(base, n++);
        continue;
      }
      float x = ang ? d6_row_angle_dev(hinge, rot_a, rot_b, i) : dot(d, u);
      JRowD lo = base, hi = base;
      lo.target = rmin((j.lo[ax] - x) / dt, 0.0f); lo.lo = 0.0f; lo.tag = base.tag | 2u;
      hi.target = rmax((j.hi[ax] - x) / dt, 0.0f); hi.hi = 0.0f; hi.lo = -INFINITY; hi.tag = base.tag | 3u;
      emit(lo, n++);
      emit(hi, n++);
    }
  }
  return n;
}

// distance_rows (solver.rs:309-330): an anchored rigid rod's equality row along the current
// anchors' direction (a compliant rod has none); and the original COM-to-COM row (solver.rs:
// 793-817), made once per tick since positions do not move during the velocity solve.
template <class Emit>
__device__ __forceinline__ uint32_t distance_rows_dev(const JointGpu& j, const BodiesV& B, float dt, Emit&& emit) {
  const uint32_t a = j.a, b = j.b;
  const float rest = j.lo[0], compliance = j.comp[0];
  if (j.flags & JF_ANCH) {
    float wa = B.inv_mass[a], wb = B.inv_mass[b];
    if (wa == 0.0f && wb == 0.0f) return 0;
    q4 qa = asq(B.rot[a]), qb = asq(B.rot[b]);
    f3 ra = qrot(qa, xyz(j.fa_p)), rb = qrot(qb, xyz(j.fb_p));
    f3 d = (xyz(B.pos[b]) + rb) - (xyz(B.pos[a]) + ra);
    float len = sqrtf(len2(d));
    if (!(len > 1e-6f)) return 0;
    f3 u = d / len;
    m3 ia = inv_inertia_world_dev(B, a, qa), ib = inv_inertia_world_dev(B, b, qb);
    f3 ca = cross(ra, u), cb = cross(rb, u);
    float k = ((wa + wb) + dot(ca, mvec(ia, ca))) + dot(cb, mvec(ib, cb));
    if (!(k > 1e-9f)) return 0;
    if (compliance > 0.0f) return 0;
    JRowD r;
    r.u = u; r.ra = ra; r.rb = rb; r.wa = wa; r.wb = wb; r.m_eff = 1.0f / k;
    r.target = 0.0f; r.lo = -INFINITY; r.hi = INFINITY; r.gamma = 0.0f; r.tag = 0; r.angular = false;
    emit(r, 0u);
    return 1;
  }
  if (compliance > 0.0f) return 0;  // a spring acts at position level only
  f3 dir = xyz(B.pos[b]) - xyz(B.pos[a]);
  float len = sqrtf(len2(dir));
  if (len < 1e-6f) return 0;
  f3 n = dir / len;
  float inv_a = B.inv_mass[a], inv_b = B.inv_mass[b];
  float inv_sum = inv_a + inv_b;
  if (inv_sum < 1e-9f) return 0;
  JRowD r;
  r.u = n; r.ra = mk3(0, 0, 0); r.rb = mk3(0, 0, 0); r.wa = inv_a; r.wb = inv_b; r.m_eff = 1.0f / inv_sum;
  r.target = 0.0f; r.lo = -INFINITY; r.hi = INFINITY; r.gamma = 0.0f; r.tag = 0; r.angular = false;
  r.legacy = true;
  r.bias = (len - rest) * (0.1f / dt);
  r.inv_sum = inv_sum;
  emit(r, 0u);
  return 1;
}
// A joint's velocity rows whatever its kind (solver.rs:655-661); a joint with a dynamic body and
// no row gets one carrier row, which puts it in the schedules for its position solve (a task of
// the reference's joint batches, which hold every active joint) and does nothing at velocity level.
template <class Emit>
__device__ __forceinline__ uint32_t joint_rows_dev(const JointGpu& j, const BodiesV& B, float dt, Emit&& emit) {
  uint32_t n = (j.flags & JF_DIST) ? distance_rows_dev(j, B, dt, emit) : d6_rows_dev(j, B, dt, emit);
  const float wa = B.inv_mass[j.a], wb = B.inv_mass[j.b];
  if (n == 0 && (wa > 0.0f || wb > 0.0f)) {
    JRowD r;
    r.u = mk3(0, 0, 0); r.ra = mk3(0, 0, 0); r.rb = mk3(0, 0, 0); r.wa = wa; r.wb = wb; r.m_eff = 1.0f;
    r.target = 0.0f; r.lo = -INFINITY; r.hi = INFINITY; r.gamma = 0.0f; r.tag = 0; r.angular = false;
    r.carrier = true;
    emit(r, 0u);
    n = 1;
  }
  return n;
}

// ---- the position solve (bodies.rs:616-873) on the bodies' global pose arrays
// Bodies::apply_position_delta / apply_orientation_delta (dynamics.rs:71-88, 207-210)
__device__ __forceinline__ void apply_position_delta_dev(const BodiesV& B, uint32_t id, f3 dp) {
  if (B.inv_mass[id] > 0.0f && vfin(dp)) { float4 P = B.pos[id]; B.pos[id] = f4(fin_v(xyz(P) + dp), P.w); }
}
__device__ __forceinline__ void apply_orientation_delta_dev(const BodiesV& B, uint32_t id, f3 dth) {
  if (B.inv_mass[id] <= 0.0f || !vfin(dth)) return;
  f3 d = fin_v(dth);
  if (len2(d) <= 1.0e-24f) return;
  q4 dq = qnormalize(mkq(d.x * 0.5f, d.y * 0.5f, d.z * 0.5f, 1.0f));
  B.rot[id] = f4q(fin_q(qnormalize(qmul(dq, asq(B.rot[id])))));
}
// turned(a, b) < SHAKE_MAX_TURN (bodies.rs:486-490, :477): 2 acos(d) < 0.5 with d = min(|w|, 1),
// w the real part of a b*. acos is decreasing and the project's acos (one rounding of a double
// evaluation) is monotone in d, so the test is d >= the least f32 that passes it, 0x3f780aa6
// (0.968912482); tests/test_oracle_joints.py checks the two forms agree on every f32 in [0.8, 1]
// (below that 2 acos(d) exceeds 1.28).
#define RP_SHAKE_COS_BITS 0x3f780aa6u
__device__ __forceinline__ bool turned_below_max(q4 a, q4 b) {
  float d = rmin(fabsf(qmul(a, qconj(b)).w), 1.0f);
  return d >= __uint_as_float(RP_SHAKE_COS_BITS);
}
// alpha_dt2 (bodies.rs:438-441)
__device__ __forceinline__ float alpha_dt2_dev(float c, float dt2) {
  c = rmax(fin0(c), 0.0f);
  return c <= 0.0f ? 0.0f : fin0(c / dt2);
}
// The error axis ax acts on at coordinate coord (bodies.rs:674-698, 786-810): locked at 0, a limit
// only while violated, a position drive's target clamped into the limit; a velocity drive leaves
// an unlimited axis free at position level. False: nothing to correct.
__device__ __forceinline__ bool row_error_dev(const JointGpu& j, int ax, float coord, float* c) {
  bool has = true;
  *c = fin0(coord - 0.0f);
  const bool lim = jaxis_lim(j.flags, ax);
  if (lim) {
    float lo = fin0(j.lo[ax]), hi = fin0(j.hi[ax]);
    if (coord < lo) *c = fin0(coord - lo);
    else if (coord > hi) *c = fin0(coord - hi);
    else has = false;
  }
  if (jaxis_drive(j.flags, ax)) {
    if (!jaxis_vel(j.flags, ax)) {
      float target = fin0(j.dtarget[ax]);
      if (lim) target = clampf(target, fin0(j.lo[ax]), fin0(j.hi[ax]));
      *c = fin0(coord - target);
      has = true;
    } else if (!lim) {
      has = false;
    }
  }
  return has;
}
// row_error for an axis with no drive: 0 when locked, the violation when limited (false: inside).
__device__ __forceinline__ bool limit_error_dev(const JointGpu& j, int ax, float coord, float* c) {
  *c = fin0(coord - 0.0f);
  if (jaxis_lim(j.flags, ax)) {
    float lo = fin0(j.lo[ax]), hi = fin0(j.hi[ax]);
    if (coord < lo) *c = fin0(coord - lo);
    else if (coord > hi) *c = fin0(coord - hi);
    else return false;
  }
  return true;
}
// The measure of rotational axis i at joint-frame rotations ra, rb (bodies.rs:796-803).
__device__ __forceinline__ float row_angle_dev(int hinge, q4 ra, q4 rb, int i, f3 u) {
  q4 q = qmul(qconj(ra), rb);
  if (q.w < 0.0f) q = qneg(q);
  f3 v = mk3(q.x, q.y, q.z);
  if (hinge == i) return fin0(2.0f * atan2_rp(comp3(v, i), q.w));
  if (hinge >= 0)
    return fin0(dot(fin_v(cross(normalize_fin(qrot(ra, unit_axis(hinge))), normalize_fin(qrot(rb, unit_axis(hinge))))), u));
  return fin0(dot(fin_v(qrot(ra, fin_v(v * 2.0f))), u));
}

// solve_d6 (bodies.rs:616-873) without the rotor rows (no armature). lam: the joint's six XPBD
// multipliers of this step (t0 t1 t2 r0 r1 r2). sa / sb: the step's start poses, for SHAKE's
// directions (when neither body turned too far) and for a damped compliant axis's change since the
// start (Kelvin-Voigt: spring and damper in one implicit row). kFull = false is the same solve for a
// joint with no compliant and no driven axis (JF_FULL clear): every alpha is 0, no axis is
// position-damped and row_error is the limit test alone -- the same operations, without the loads
// and branches of the other cases (a shorter dependent chain in the position pass).
template <bool kFull>
__device__ __forceinline__ void solve_d6_dev(const JointGpu& j, float* lam, const BodiesV& B, float dt, f3 sa_p,
                                             q4 sa_q, f3 sb_p, q4 sb_q) {
  const uint32_t A = j.a, Bb = j.b;
  const float wa = fin0(B.inv_mass[A]), wb = fin0(B.inv_mass[Bb]);
  const float dt2 = kFull ? rmax(dt * dt, 1.0e-12f) : 0.0f;
  const bool shake = turned_below_max(sa_q, asq(B.rot[A])) && turned_below_max(sb_q, asq(B.rot[Bb]));
  // SHAKE's directions: axis i of the start frame, normalize_fin(qrot(r0, e_i)), made where used
  f3 la0 = mk3(0, 0, 0), lb0 = mk3(0, 0, 0);
  m3 ia0 = mzero(), ib0 = mzero();
  const uint32_t flags = j.flags;
  const q4 fa_q = asq(j.fa_q), fb_q = asq(j.fb_q);
  const f3 fa_p = xyz(j.fa_p), fb_p = xyz(j.fb_p);
  const q4 r0 = qmul(sa_q, fa_q);
  if (shake) {
    la0 = fin_v(qrot(sa_q, fa_p));
    lb0 = fin_v(qrot(sb_q, fb_p));
    ia0 = world_inertia(sa_q, ld_m3(B.inv_I, A));
    ib0 = world_inertia(sb_q, ld_m3(B.inv_I, Bb));
  }
  const float bias_vel = 0.0f;
  for (int i = 0; i < 3; ++i) {
    if (!jaxis_on(flags, i)) continue;
    f3 pap = xyz(B.pos[A]), pbp = xyz(B.pos[Bb]);
    q4 paq = asq(B.rot[A]), pbq = asq(B.rot[Bb]);
    f3 u = normalize_fin(qrot(qmul(paq, fa_q), unit_axis(i)));
    if (vzero(u)) continue;
    f3 xa = fin_v(pap + qrot(paq, fa_p)), xb = fin_v(pbp + qrot(pbq, fb_p));
    f3 d = fin_v(xb - xa);
    f3 un, lever_a, lever_b;
    m3 iaw, ibw;
    if (shake) { un = normalize_fin(qrot(r0, unit_axis(i))); lever_a = la0; lever_b = lb0; iaw = ia0; ibw = ib0; }
    else {
      un = u; lever_a = xa - pap; lever_b = xb - pbp;
      iaw = inv_inertia_world_dev(B, A, paq); ibw = inv_inertia_world_dev(B, Bb, pbq);
    }
    float coord = fin0(dot(d, u));
    float c;
    if (kFull) {
      if (!row_error_dev(j, i, coord, &c)) continue;
    } else if (!limit_error_dev(j, i, coord, &c)) continue;
    f3 ra_u = fin_v(cross(lever_a, un)), rb_u = fin_v(cross(lever_b, un));
    float w_rot_a = fin0(dot(ra_u, mvec(iaw, ra_u)));
    float w_rot_b = fin0(dot(rb_u, mvec(ibw, rb_u)));
    float ws = fin0(((wa + wb) + w_rot_a) + w_rot_b);
    float alpha = kFull ? alpha_dt2_dev(j.comp[i], dt2) : 0.0f;
    float denom = fin0(ws + alpha);
    if (denom <= 0.0f) continue;
    c = fin0(c + fin0(bias_vel * dt));
    float lambda_old = fin0(lam[i]);
    float dl;
    if (kFull && position_damped_dev(j, i)) {
      f3 u0 = normalize_fin(qrot(qmul(sa_q, fa_q), unit_axis(i)));
      f3 d0 = fin_v((sb_p + qrot(sb_q, fb_p)) - (sa_p + qrot(sa_q, fa_p)));
      float gamma = fin0(j.comp[i] * j.damp[i] / dt);
      float dc = fin0(coord - dot(d0, u0));
      dl = fin0(-((c + fin0(alpha * lambda_old)) + fin0(gamma * dc)) / fin0((1.0f + gamma) * ws + alpha));
    } else {
      dl = fin0(-(c + fin0(alpha * lambda_old)) / denom);
    }
    lam[i] = fin0(lambda_old + dl);
    apply_position_delta_dev(B, A, fin_v((-un) * fin0(dl * wa)));
    apply_position_delta_dev(B, Bb, fin_v(un * fin0(dl * wb)));
    apply_orientation_delta_dev(B, A, fin_v((-mvec(iaw, ra_u)) * dl));
    apply_orientation_delta_dev(B, Bb, fin_v(mvec(ibw, rb_u) * dl));
  }
  const int hinge = joint_hinge(flags);
  for (int i = 0; i < 3; ++i) {
    const int ax = 3 + i;
    if (!jaxis_on(flags, ax)) continue;
    q4 paq = asq(B.rot[A]), pbq = asq(B.rot[Bb]);
    q4 ra = qmul(paq, fa_q), rb = qmul(pbq, fb_q);
    f3 u = normalize_fin(qrot(ra, unit_axis(i)));
    if (vzero(u)) continue;
    float angle = row_angle_dev(hinge, ra, rb, i, u);
    f3 un;
    m3 iaw, ibw;
    if (shake) { un = normalize_fin(qrot(r0, unit_axis(i))); iaw = ia0; ibw = ib0; }
    else { un = u; iaw = inv_inertia_world_dev(B, A, paq); ibw = inv_inertia_world_dev(B, Bb, pbq); }
    float c;
    if (kFull) {
      if (!row_error_dev(j, ax, angle, &c)) continue;
    } else if (!limit_error_dev(j, ax, angle, &c)) continue;
    float ws = fin0(dot(un, mvec(iaw, un)) + dot(un, mvec(ibw, un)));
    float alpha = kFull ? alpha_dt2_dev(j.comp[ax], dt2) : 0.0f;
    float denom = fin0(ws + alpha);
    if (denom <= 0.0f) continue;
    c = fin0(c + fin0(bias_vel * dt));
    float lambda_old = fin0(lam[ax]);
    float dl;
    if (kFull && position_damped_dev(j, ax)) {
      q4 ra0 = qmul(sa_q, fa_q), rb0 = qmul(sb_q, fb_q);
      f3 u0 = normalize_fin(qrot(ra0, unit_axis(i)));
      float angle0 = row_angle_dev(hinge, ra0, rb0, i, u0);
      float gamma = fin0(j.comp[ax] * j.damp[ax] / dt);
      float dc = fin0(angle - angle0);
      dl = fin0(-((c + fin0(alpha * lambda_old)) + fin0(gamma * dc)) / fin0((1.0f + gamma) * ws + alpha));
    } else {
      dl = fin0(-(c + fin0(alpha * lambda_old)) / denom);
    }
    lam[ax] = fin0(lambda_old + dl);
    apply_orientation_delta_dev(B, A, fin_v((-mvec(iaw, un)) * dl));
    apply_orientation_delta_dev(B, Bb, fin_v(mvec(ibw, un) * dl));
  }
}

// ---- host side (joints.cu)
struct StepCtx;
// Reference islands: joint unions (both bodies dynamic) into uf and the island marks.
void joints_ref_islands(WorldGpu& W, uint32_t* uf, uint32_t* root_mark, bool unions, cudaStream_t st);
// Row counts and offsets per joint; returns the total number of joint velocity rows.
uint32_t joints_count_rows(WorldGpu& W, float dt, const BodiesV& B, cudaStream_t st);
// Joint rows at R[base .. base + njr): geometry, bounds, warm start from the joint cache, flags;
// then the joint-row unions into the solve union-find uf.
void joints_build_rows(WorldGpu& W, float dt, const BodiesV& B, const RowsV& R, uint32_t base, float* acc_jn,
                       float2* acc_jt, uint32_t* uf, cudaStream_t st);
// The solve-island root of every joint row (after every union is in).
void joints_row_roots(WorldGpu& W, const RowsV& R, uint32_t base, uint32_t njr, uint32_t* uf, uint32_t* row_root,
                      cudaStream_t st);
// The joint warm cache (solver.rs:946-952) from the accumulated impulses.
void joints_store_warm(WorldGpu& W, const RowsV& R, uint32_t base, const float* acc_jn, cudaStream_t st);
// Bodies in joints count as constrained (step.rs:160-170).
void joints_mark_constrained(WorldGpu& W, uint8_t* constrained, cudaStream_t st);

// SHAKE_MAX_TURN.cos() (bodies.rs:520) as the project's cosine gives it: 0.87758255
// (tests/test_oracle_joints.py checks the oracle's value has these bits).
#define RP_SHAKE_MAX_TURN_COS_BITS 0x3f60a940u
// solve_distance_row (bodies.rs:501-548): the original COM-to-COM rod, corrected along the
// start-of-step direction when it is within SHAKE_MAX_TURN of the current one. lam: its multiplier.
__device__ __forceinline__ void solve_distance_row_dev(const JointGpu& j, float* lam, const BodiesV& B, float dt2,
                                                       f3 sa_p, f3 sb_p) {
  const uint32_t ia = j.a, ib = j.b;
  const float wa = B.inv_mass[ia], wb = B.inv_mass[ib];
  const float w_sum = fin0(wa + wb);
  if (w_sum <= 0.0f) return;
  f3 d = xyz(B.pos[ib]) - xyz(B.pos[ia]);
  float l2 = len2(d);
  if (!fin(l2) || l2 <= 1.0e-20f) return;
  float len = sqrtf(l2);
  if (len <= 1.0e-6f) return;
  f3 n_cur = normalize_fin(d / len);
  if (vzero(n_cur)) return;
  f3 n = n_cur;
  f3 n0 = normalize_fin(sb_p - sa_p);
  if (!vzero(n0) && dot(n0, n_cur) > __uint_as_float(RP_SHAKE_MAX_TURN_COS_BITS)) n = n0;
  const float compliance = j.comp[0];
  float c_val = fin0(len - fin0(j.lo[0]));
  float alpha = compliance <= 0.0f ? 0.0f : fin0(rmax(fin0(compliance), 0.0f) / dt2);
  float denom = fin0(w_sum + alpha);
  if (denom <= 0.0f) return;
  float lambda_old = fin0(lam[0]);
  float lambda = fin0(-(c_val + fin0(alpha * lambda_old)) / (denom * dot(n, n_cur)));
  if (fabsf(lambda) <= 1.0e-9f) return;
  lam[0] = fin0(lambda_old + lambda);
  apply_position_delta_dev(B, ia, fin_v((-n) * fin0(lambda * wa)));
  apply_position_delta_dev(B, ib, fin_v(n * fin0(lambda * wb)));
}
// solve_distance_anchored (bodies.rs:557-614): C = |x_b - x_a| - rest on the current anchors, along
// the start-of-step direction with start-of-step lever arms and inertias over the mixed Jacobian
// product (current-iterate directions when a body turned too far or the mixed product falls below
// half the start-of-step one); a damped compliant rod's spring and damper in one Kelvin-Voigt row.
__device__ __forceinline__ void solve_distance_anchored_dev(const JointGpu& j, float* lam, const BodiesV& B, float dt,
                                                            float dt2, f3 sa_p, q4 sa_q, f3 sb_p, q4 sb_q) {
  const uint32_t ia = j.a, ib = j.b;
  const float wa = fin0(B.inv_mass[ia]), wb = fin0(B.inv_mass[ib]);
  if (wa + wb <= 0.0f) return;
  const f3 la = xyz(j.fa_p), lb = xyz(j.fb_p);
  const float rest = j.lo[0], compliance = j.comp[0], damping = j.damp[0];
  f3 pap = xyz(B.pos[ia]), pbp = xyz(B.pos[ib]);
  q4 paq = asq(B.rot[ia]), pbq = asq(B.rot[ib]);
  f3 ra = fin_v(qrot(paq, la)), rb = fin_v(qrot(pbq, lb));
  f3 d = fin_v((pbp + rb) - (pap + ra));
  float len = sqrtf(len2(d));
  if (!fin(len) || len <= 1.0e-6f) return;
  f3 n_cur = normalize_fin(d / len);
  if (vzero(n_cur)) return;
  float c_val = fin0(len - fin0(rest));
  float alpha = compliance <= 0.0f ? 0.0f : fin0(rmax(fin0(compliance), 0.0f) / dt2);
  f3 n = n_cur, ga, gb;
  float wgen = 0.0f;
  bool shake = false;
  if (turned_below_max(sa_q, paq) && turned_below_max(sb_q, pbq)) {
    f3 ra0 = qrot(sa_q, la), rb0 = qrot(sb_q, lb);
    f3 n0 = normalize_fin((sb_p + rb0) - (sa_p + ra0));
    if (!vzero(n0)) {
      m3 ia0 = world_inertia(sa_q, ld_m3(B.inv_I, ia)), ib0 = world_inertia(sb_q, ld_m3(B.inv_I, ib));
      f3 ga0 = mvec(ia0, cross(ra0, n0)), gb0 = mvec(ib0, cross(rb0, n0));
      float w_sym = ((wa + wb) + dot(cross(ra0, n0), ga0)) + dot(cross(rb0, n0), gb0);
      float w_mix = (((wa + wb) * dot(n_cur, n0)) + dot(cross(ra, n_cur), ga0)) + dot(cross(rb, n_cur), gb0);
      if (fin(w_mix) && w_mix >= 0.5f * w_sym) { shake = true; n = n0; ga = ga0; gb = gb0; wgen = w_mix; }
    }
  }
  if (!shake) {
    m3 iaw = inv_inertia_world_dev(B, ia, paq), ibw = inv_inertia_world_dev(B, ib, pbq);
    f3 ca = cross(ra, n_cur), cb = cross(rb, n_cur);
    wgen = ((wa + wb) + dot(ca, mvec(iaw, ca))) + dot(cb, mvec(ibw, cb));
    n = n_cur; ga = mvec(iaw, ca); gb = mvec(ibw, cb);
  }
  float denom = fin0(wgen + alpha);
  if (!(denom > 0.0f)) return;
  float lambda_old = fin0(lam[0]);
  float dl;
  if (compliance > 0.0f && damping > 0.0f) {
    float len0 = sqrtf(len2((sb_p + qrot(sb_q, lb)) - (sa_p + qrot(sa_q, la))));
    float gamma = fin0(compliance * damping / dt);
    dl = fin0(-((c_val + fin0(alpha * lambda_old)) + fin0(gamma * fin0(len - len0))) / fin0((1.0f + gamma) * wgen + alpha));
  } else {
    dl = fin0(-(c_val + fin0(alpha * lambda_old)) / denom);
  }
  if (fabsf(dl) <= 1.0e-12f) return;
  lam[0] = fin0(lambda_old + dl);
  apply_position_delta_dev(B, ia, fin_v((-n) * fin0(dl * wa)));
  apply_position_delta_dev(B, ib, fin_v(n * fin0(dl * wb)));
  apply_orientation_delta_dev(B, ia, fin_v((-ga) * dl));
  apply_orientation_delta_dev(B, ib, fin_v(gb * dl));
}
// The position solve of joint j: a distance joint's row; for a D6 joint the full path when it has
// a compliant or driven axis, the locked-and-limited one otherwise.
__device__ __forceinline__ void solve_joint_pos(const JointGpu& j, float* lam, const BodiesV& B, float dt, f3 sa_p,
                                                q4 sa_q, f3 sb_p, q4 sb_q) {
  if (j.flags & JF_DIST) {
    const float dt2 = rmax(dt * dt, 1.0e-12f);
    if (j.flags & JF_ANCH) solve_distance_anchored_dev(j, lam, B, dt, dt2, sa_p, sa_q, sb_p, sb_q);
    else solve_distance_row_dev(j, lam, B, dt2, sa_p, sb_p);
  } else if (j.flags & JF_FULL) {
    solve_d6_dev<true>(j, lam, B, dt, sa_p, sa_q, sb_p, sb_q);
  } else {
    solve_d6_dev<false>(j, lam, B, dt, sa_p, sa_q, sb_p, sb_q);
  }
}

}  // namespace rp
