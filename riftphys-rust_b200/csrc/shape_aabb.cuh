// shape_aabb.cuh -- a collider's world AABB as the reference stores it, shared by the tick's
// broadphase (step_front.cu) and the scene queries (query.cu).
#pragma once
#include "rp_narrow.cuh"

namespace rp {

// aabb_of (shape.rs:7-56) with Aabb::new's 1e-6 quantisation (aabb.rs:21-26)
__device__ __forceinline__ void aabb_of(uint32_t kind, float4 d, f3 p, q4 q, f3* mn, f3* mx) {
  f3 he;
  if (kind == SH_SPHERE) he = splat(fabsf(d.x));
  else if (kind == SH_BOX) {
    m3 r = mfrom_quat(q);
    m3 ar = mcols(vabs(r.c0), vabs(r.c1), vabs(r.c2));
    he = mvec(ar, mk3(fabsf(d.x), fabsf(d.y), fabsf(d.z)));
  } else {
    f3 axis = qrot(q, mk3(0, 1, 0)) * fabsf(d.y);
    he = vabs(axis) + splat(fabsf(d.x));
  }
  f3 a = p - he, b = p + he;
  a = mk3(qf32(a.x), qf32(a.y), qf32(a.z));
  b = mk3(qf32(b.x), qf32(b.y), qf32(b.z));
  *mn = vmin(a, b);
  *mx = vmax(a, b);
}

}  // namespace rp
