// hf_cells.cuh -- the heightfield's cells seen from a query box, for the device queries:
// Heightfield::query_aabb (riftphys-world/src/terrain.rs:300-358) returns, for the grid cells
// under the box widened by one cell each way, two triangles per cell, rows of z outside, x inside.
// hf_window gives that cell window; hf_tri builds the k-th triangle of it.
#pragma once
#include "rp_narrow.cuh"

namespace rp {

struct HfDev { const float* h; uint32_t nx, nz; float sx, sz, ox, oz, min_y, max_y; };

// false when the box misses the height range (one unit of slack) or the grid has no cell
__device__ __forceinline__ bool hf_window(const HfDev& hf, f3 qmn, f3 qmx, long long* gx0, long long* gx1,
                                          long long* gz0, long long* gz1) {
  const int nx = (int)hf.nx, nz = (int)hf.nz;
  if (nx < 2 || nz < 2 || qmn.y > hf.max_y + 1.0f || qmx.y < hf.min_y - 1.0f) return false;
  auto toi = [](float f) -> long long {  // Rust's saturating f32 -> i32 cast
    if (isnan(f)) return 0;
    if (f >= 2147483647.0f) return 2147483647;
    if (f <= -2147483648.0f) return -2147483648LL;
    return (long long)f;
  };
  auto cl = [](long long v, long long lo, long long hi) { return v < lo ? lo : (v > hi ? hi : v); };
  *gx0 = cl(toi(floorf((qmn.x - hf.ox) / hf.sx)) - 1, 0, nx - 2);
  *gx1 = cl(toi(ceilf((qmx.x - hf.ox) / hf.sx)) + 1, 0, nx - 2);
  *gz0 = cl(toi(floorf((qmn.z - hf.oz) / hf.sz)) - 1, 0, nz - 2);
  *gz1 = cl(toi(ceilf((qmx.z - hf.oz) / hf.sz)) + 1, 0, nz - 2);
  return true;
}
// triangle k of the window starting at (gx0, gz0), wx cells wide: cell k / 2, its lower-left
// triangle (p00, p01, p10) for even k, the upper-right one (p10, p01, p11) for odd k
__device__ __forceinline__ void hf_tri(const HfDev& hf, long long gx0, unsigned long long wx, long long gz0,
                                       unsigned long long k, Tri* t) {
  const unsigned long long cell = k >> 1;
  const long long gz = gz0 + (long long)(cell / wx), gx = gx0 + (long long)(cell % wx);
  auto H = [&](long long x, long long z) { return hf.h[(size_t)x + (size_t)z * hf.nx]; };
  const float x0 = (float)gx * hf.sx + hf.ox, x1 = x0 + hf.sx;
  const float z0 = (float)gz * hf.sz + hf.oz, z1 = z0 + hf.sz;
  const f3 p00 = mk3(x0, H(gx, gz), z0), p10 = mk3(x1, H(gx + 1, gz), z0);
  const f3 p01 = mk3(x0, H(gx, gz + 1), z1), p11 = mk3(x1, H(gx + 1, gz + 1), z1);
  if (k & 1ull) { t->a = p10; t->b = p01; t->c = p11; }
  else { t->a = p00; t->b = p01; t->c = p10; }
}

}  // namespace rp
