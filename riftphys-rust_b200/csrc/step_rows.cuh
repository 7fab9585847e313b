// step_rows.cuh -- the row and body views the solve kernels share (step_solve.cu, joints.cu):
// row flag bits, the structure-of-arrays row view, the body view, 3x3 loads, union-find.
#pragma once
#include "step_internal.cuh"

namespace rp {

// row flag bits
// RF_WA / RF_WB: the row writes body A / B. RF_RA / RF_RB: the row only reads that side, a sleeping
// body in a joint, whose joint rows move it in the same sweep: it orders the row like a write
// (levels, solve islands) without receiving impulses. RF_JOINT: a joint velocity row (RF_JANG:
// angular; RF_JWARM: warm-started from the previous tick; RF_JFIRST: the joint's first row, which
// carries the joint's position solve in the position pass; RF_JLEG: the original distance row,
// impulse -(v_rel + bias) / inv_sum on the linear velocities, bias in t1.w, inv_sum in rb.w;
// RF_JNULL: the carrier row of a joint with no velocity row, which puts the joint in the schedules
// for its position solve and does nothing in the velocity solve).
enum : uint32_t {
  RF_TERRAIN = 1, RF_TOI = 4, RF_WA = 8, RF_WB = 16, RF_RA = 32, RF_RB = 64,
  RF_JOINT = 128, RF_JANG = 256, RF_JWARM = 512, RF_JFIRST = 1024, RF_JLEG = 2048, RF_JNULL = 4096
};
#define RF_TA (RF_WA | RF_RA)
#define RF_TB (RF_WB | RF_RB)

__device__ __forceinline__ m3 ld_m3(const float* p, uint32_t i) {
  const float* q = p + 9 * (size_t)i;
  return mcols(mk3(q[0], q[1], q[2]), mk3(q[3], q[4], q[5]), mk3(q[6], q[7], q[8]));
}
__device__ __forceinline__ void st_m3(float* p, uint32_t i, const m3& m) {
  float* q = p + 9 * (size_t)i;
  q[0] = m.c0.x; q[1] = m.c0.y; q[2] = m.c0.z; q[3] = m.c1.x; q[4] = m.c1.y; q[5] = m.c1.z;
  q[6] = m.c2.x; q[7] = m.c2.y; q[8] = m.c2.z;
}

// ------------------------------------------------------------------ islands (islands.rs:27-93)
__device__ __forceinline__ uint32_t uf_find(uint32_t* p, uint32_t x) {
  volatile uint32_t* vp = p;
  while (true) {
    uint32_t px = vp[x];
    if (px == x) return x;
    uint32_t ppx = vp[px];
    if (ppx != px) atomicCAS(&p[x], px, ppx);  // path halving
    x = px;
  }
}
// Union by hooking the larger root under the smaller: each component's root is its least body.
__device__ __forceinline__ void uf_union(uint32_t* p, uint32_t a, uint32_t b) {
  while (true) {
    uint32_t ra = uf_find(p, a), rb = uf_find(p, b);
    if (ra == rb) return;
    if (ra > rb) { uint32_t t = ra; ra = rb; rb = t; }
    if (atomicCAS(&p[rb], rb, ra) == rb) return;
  }
}
struct RowsV {
  uint2* ab; uint32_t* flags; float2* inv; float4 *ra, *rb, *n, *t1, *t2, *mu, *la;
};
struct BodiesV {
  float4 *pos, *rot, *lin, *ang;
  const float* inv_mass; const float* Iw; const float* inv_I; const uint8_t* awake; const uint8_t* dyn;
};

}  // namespace rp
