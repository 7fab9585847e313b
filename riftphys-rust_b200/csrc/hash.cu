// hash.cu -- World::step_hash (riftphys-world/src/world/provenance.rs:6-24 and hash_carried,
// world.rs:882-909) on the GPU: the byte stream is written in place by one thread per record,
// then hashed with BLAKE3 (`blake3` crate 1.8.2, Cargo.lock:267-269; algorithm from the published
// BLAKE3 specification): one thread compresses each 1 KiB chunk, then parent nodes are merged
// pairwise, level by level -- the left-complete tree the specification defines (an odd last node
// moves up a level unchanged). BLAKE3 is integer-ALU work (32-bit add / xor / rotate).
//
// Stream layout: epoch u64 | rng state u64 | BLAKE3("") (the empty schedule digest) |
//   per body: index u32, pos xyz, rot xyzw, lin xyz, ang xyz (canonical f32 bits) |
//   warm keys u64 | per key: 4 x u32, count u32, per entry la xyz, jn, jt xyz |
//   warm patches u64 0 | warm joints u64 | per entry: joint u32, rows u32, per row tag u8 +
//   impulse | rotors u64 0 |
//   last_lin_vel count u64 + xyz each | awake count u64 + u8 each | sleep ticks count u64 + u16 each.
#include <cstring>
#include <mutex>
#include <stdexcept>

#include <cub/device/device_scan.cuh>

#include "step_internal.cuh"

namespace rp {

__constant__ uint32_t c_iv[8] = {0x6A09E667u, 0xBB67AE85u, 0x3C6EF372u, 0xA54FF53Au,
                                 0x510E527Fu, 0x9B05688Cu, 0x1F83D9ABu, 0x5BE0CD19u};

__device__ __forceinline__ uint32_t rotr(uint32_t x, int n) { return __funnelshift_r(x, x, n); }
#define B3G(a, b, c, d, x, y)        \
  a = a + b + x; d = rotr(d ^ a, 16); \
  c = c + d; b = rotr(b ^ c, 12);     \
  a = a + b + y; d = rotr(d ^ a, 8);  \
  c = c + d; b = rotr(b ^ c, 7);

// The compression function: 7 rounds, message words permuted between rounds by the
// specification's fixed permutation (2, 6, 3, 10, 7, 0, 4, 13, 1, 11, 12, 5, 9, 14, 15, 8).
__device__ void b3_compress(const uint32_t cv[8], const uint32_t blk[16], uint64_t counter, uint32_t blen,
                            uint32_t flags, uint32_t out[8]) {
  uint32_t s0 = cv[0], s1 = cv[1], s2 = cv[2], s3 = cv[3], s4 = cv[4], s5 = cv[5], s6 = cv[6], s7 = cv[7];
  uint32_t s8 = c_iv[0], s9 = c_iv[1], s10 = c_iv[2], s11 = c_iv[3];
  uint32_t s12 = (uint32_t)counter, s13 = (uint32_t)(counter >> 32), s14 = blen, s15 = flags;
  uint32_t m[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) m[i] = blk[i];
#pragma unroll
  for (int r = 0; r < 7; ++r) {
    B3G(s0, s4, s8, s12, m[0], m[1]);
    B3G(s1, s5, s9, s13, m[2], m[3]);
    B3G(s2, s6, s10, s14, m[4], m[5]);
    B3G(s3, s7, s11, s15, m[6], m[7]);
    B3G(s0, s5, s10, s15, m[8], m[9]);
    B3G(s1, s6, s11, s12, m[10], m[11]);
    B3G(s2, s7, s8, s13, m[12], m[13]);
    B3G(s3, s4, s9, s14, m[14], m[15]);
    if (r < 6) {
      uint32_t t[16] = {m[2], m[6], m[3], m[10], m[7], m[0], m[4], m[13], m[1], m[11], m[12], m[5], m[9], m[14], m[15], m[8]};
#pragma unroll
      for (int i = 0; i < 16; ++i) m[i] = t[i];
    }
  }
  out[0] = s0 ^ s8; out[1] = s1 ^ s9; out[2] = s2 ^ s10; out[3] = s3 ^ s11;
  out[4] = s4 ^ s12; out[5] = s5 ^ s13; out[6] = s6 ^ s14; out[7] = s7 ^ s15;
}
enum : uint32_t { CHUNK_START = 1, CHUNK_END = 2, PARENT = 4, ROOT = 8 };

// One thread per 1024-byte chunk: its chaining value; a single-chunk input is finalised as root.
__global__ void k_b3_chunks(const uint8_t* __restrict__ data, uint64_t len, uint32_t nch, uint32_t* cvs, uint32_t* root) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nch) return;
  uint64_t base = (uint64_t)c * 1024;
  uint64_t clen = len - base < 1024 ? len - base : 1024;
  uint32_t nblocks = clen == 0 ? 1 : (uint32_t)((clen + 63) / 64);
  uint32_t cv[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) cv[i] = c_iv[i];
  for (uint32_t b = 0; b < nblocks; ++b) {
    uint32_t blk[16];
    const uint32_t* w = reinterpret_cast<const uint32_t*>(data + base + 64 * (uint64_t)b);
#pragma unroll
    for (int i = 0; i < 16; ++i) blk[i] = w[i];  // zero-padded past len (little-endian words)
    uint32_t blen = b + 1 == nblocks ? (uint32_t)(clen - 64 * (uint64_t)b) : 64u;
    uint32_t flags = (b == 0 ? CHUNK_START : 0u) | (b + 1 == nblocks ? CHUNK_END : 0u);
    if (nch == 1 && b + 1 == nblocks) flags |= ROOT;
    uint32_t o[8];
    b3_compress(cv, blk, c, blen, flags, o);
#pragma unroll
    for (int i = 0; i < 8; ++i) cv[i] = o[i];
  }
  if (nch == 1) {
    for (int i = 0; i < 8; ++i) root[i] = cv[i];
  } else {
    for (int i = 0; i < 8; ++i) cvs[8 * c + i] = cv[i];
  }
}
// One tree level: node t of the next level is parent(2t, 2t+1), or node 2t carried up.
__global__ void k_b3_parents(uint32_t n_in, const uint32_t* __restrict__ in, uint32_t* out, uint32_t* root) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t n_out = (n_in + 1) / 2;
  if (t >= n_out) return;
  if (2 * t + 1 < n_in) {
    uint32_t blk[16];
    for (int i = 0; i < 8; ++i) { blk[i] = in[16 * t + i]; blk[8 + i] = in[16 * t + 8 + i]; }
    uint32_t cv[8];
    for (int i = 0; i < 8; ++i) cv[i] = c_iv[i];
    uint32_t o[8];
    b3_compress(cv, blk, 0, 64, PARENT | (n_in == 2 ? ROOT : 0u), o);
    uint32_t* dst = n_in == 2 ? root : out + 8 * t;
    for (int i = 0; i < 8; ++i) dst[i] = o[i];
  } else {
    for (int i = 0; i < 8; ++i) out[8 * t + i] = in[16 * t + i];
  }
}

// ---- stream writers
__device__ __forceinline__ void put32(uint8_t* p, uint32_t v) {
  p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}
__device__ __forceinline__ void put64(uint8_t* p, uint64_t v) { put32(p, (uint32_t)v); put32(p + 4, (uint32_t)(v >> 32)); }
__global__ void k_h_bodies(uint32_t nb, const float4* __restrict__ pos, const float4* __restrict__ rot,
                           const float4* __restrict__ lin, const float4* __restrict__ ang, uint8_t* out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  uint8_t* p = out + 56 * (size_t)i;
  float4 a = pos[i], q = rot[i], l = lin[i], w = ang[i];
  put32(p, i);
  put32(p + 4, canon_bits(a.x)); put32(p + 8, canon_bits(a.y)); put32(p + 12, canon_bits(a.z));
  put32(p + 16, canon_bits(q.x)); put32(p + 20, canon_bits(q.y)); put32(p + 24, canon_bits(q.z)); put32(p + 28, canon_bits(q.w));
  put32(p + 32, canon_bits(l.x)); put32(p + 36, canon_bits(l.y)); put32(p + 40, canon_bits(l.z));
  put32(p + 44, canon_bits(w.x)); put32(p + 48, canon_bits(w.y)); put32(p + 52, canon_bits(w.z));
}
__global__ void k_h_warm_flags(uint32_t n, const uint4* __restrict__ k, uint32_t* flag) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  bool first = e == 0;
  if (!first) { uint4 a = k[e], b = k[e - 1]; first = !(a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w); }
  flag[e] = first ? 1u : 0u;
}
// Entry e of group g sits after g+1 group headers (20 bytes) and e entries (28 bytes).
__global__ void k_h_warm(uint32_t n, const uint4* __restrict__ k, const float4* __restrict__ wa,
                         const float4* __restrict__ wb, const uint32_t* __restrict__ flag, const uint32_t* __restrict__ gs,
                         uint8_t* out, uint32_t base = 0) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  uint32_t g = gs[e] + flag[e] - 1;
  if (flag[e]) {
    uint32_t cnt = 1;
    while (e + cnt < n && !flag[e + cnt]) cnt++;
    uint8_t* h = out + 20 * (size_t)g + 28 * (size_t)e;
    uint4 key = k[e];
    // base: the first body of the hashed world (batched worlds hash with their own 0-based ids)
    uint32_t kb = key.y == 0xFFFFFFFFu ? key.y : key.y - base;
    put32(h, key.x - base); put32(h + 4, kb); put32(h + 8, key.z); put32(h + 12, key.w); put32(h + 16, cnt);
  }
  uint8_t* p = out + 20 * (size_t)(g + 1) + 28 * (size_t)e;
  float4 a = wa[e], b = wb[e];
  put32(p, canon_bits(a.x)); put32(p + 4, canon_bits(a.y)); put32(p + 8, canon_bits(a.z));
  put32(p + 12, canon_bits(a.w));
  put32(p + 16, canon_bits(b.x)); put32(p + 20, canon_bits(b.y)); put32(p + 24, canon_bits(b.z));
}
__global__ void k_h_tail(uint32_t nb, uint32_t cap, const float4* __restrict__ last, const uint8_t* __restrict__ awake,
                         const uint16_t* __restrict__ ticks, uint8_t* out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  // [u64 nb][12 nb][u64 cap][cap][u64 cap][2 cap]
  if (i == 0) put64(out, nb);
  if (i < nb) {
    float4 v = last[i];
    uint8_t* p = out + 8 + 12 * (size_t)i;
    put32(p, canon_bits(v.x)); put32(p + 4, canon_bits(v.y)); put32(p + 8, canon_bits(v.z));
  }
  uint8_t* a = out + 8 + 12 * (size_t)nb;
  if (i == 0) put64(a, cap);
  if (i < cap) a[8 + i] = awake[i];
  uint8_t* t = a + 8 + cap;
  if (i == 0) put64(t, cap);
  if (i < cap) { uint16_t v = ticks[i]; t[8 + 2 * i] = (uint8_t)v; t[9 + 2 * i] = (uint8_t)(v >> 8); }
}

// warm_joints (hash_carried, world.rs:895-900), entries in joint order. Joints [j0, j0 + n) of a
// batch's world hash with ids j - j0 (the arrays passed start at j0).
__global__ void k_hj_sizes(uint32_t n, const uint32_t* __restrict__ jw_n, uint32_t* sz, uint32_t* has) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  uint32_t c = jw_n[j];
  bool h = c != 0xFFFFFFFFu;
  has[j] = h ? 1u : 0u;
  sz[j] = h ? 8u + 5u * c : 0u;
}
__global__ void k_hj_write(uint32_t n, const uint32_t* __restrict__ jw_n, const uint8_t* __restrict__ tag,
                           const float* __restrict__ lam, const uint32_t* __restrict__ off, uint8_t* out) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  uint32_t c = jw_n[j];
  if (c == 0xFFFFFFFFu) return;
  uint8_t* p = out + off[j];
  put32(p, j);
  put32(p + 4, c);
  for (uint32_t k = 0; k < c; ++k) {
    p[8 + 5 * k] = tag[kJointRows * (size_t)j + k];
    put32(p + 9 + 5 * k, canon_bits(lam[kJointRows * (size_t)j + k]));
  }
}
// Sizes the joint section of joints [j0, j0 + n): bytes of its entries and their count.
static void joint_section(WorldGpu& W, uint32_t j0, uint32_t n, uint32_t* sz, uint32_t* off, uint32_t* has,
                          uint32_t* pos, uint64_t* bytes, uint64_t* count, cudaStream_t st) {
  *bytes = 0; *count = 0;
  if (!n) return;
  const int T = 256;
  k_hj_sizes<<<(n + T - 1) / T, T, 0, st>>>(n, W.jw_n.p + j0, sz, has); RP_COUNT_LAUNCH(1);
  *bytes = exclusive_scan_total(*W.s_, sz, off, n, st);
  *count = exclusive_scan_total(*W.s_, has, pos, n, st);
}
static void joint_write(WorldGpu& W, uint32_t j0, uint32_t n, const uint32_t* off, uint8_t* out, cudaStream_t st) {
  if (!n) return;
  const int T = 256;
  k_hj_write<<<(n + T - 1) / T, T, 0, st>>>(n, W.jw_n.p + j0, W.jw_tag.p + kJointRows * (size_t)j0, W.jw_lam.p + kJointRows * (size_t)j0,
                                             off, out); RP_COUNT_LAUNCH(1);
}

void WorldGpu::step_hash(uint8_t out32[32]) {
  upload_joints();
  Scratch& S = *s_;
  cudaStream_t st = stream_;
  const int T = 256;
  uint32_t cap = cap_b_ > nb_ ? cap_b_ : nb_;
  // number of distinct warm keys
  S.woff.ensure(n_warm + 1); S.wpos.ensure(n_warm + 1);
  uint32_t nkeys = 0;
  if (n_warm) {
    k_h_warm_flags<<<(n_warm + T - 1) / T, T, 0, st>>>(n_warm, warm_key.p, S.woff.p); RP_COUNT_LAUNCH(1);
    nkeys = exclusive_scan_total(S, S.woff.p, S.wpos.p, n_warm, st);
  }
  const uint32_t nj = num_joints();
  uint64_t jbytes = 0, jcount = 0;
  S.jh_sz.ensure(nj + 1); S.jh_off.ensure(nj + 1); S.jh_has.ensure(nj + 1); S.jh_pos.ensure(nj + 1);
  joint_section(*this, 0, nj, S.jh_sz.p, S.jh_off.p, S.jh_has.p, S.jh_pos.p, &jbytes, &jcount, st);
  uint64_t off_bodies = 48;
  uint64_t off_warm = off_bodies + 56ull * nb_;
  uint64_t off_joints = off_warm + 8 + 20ull * nkeys + 28ull * n_warm + 8;
  uint64_t off_tail = off_joints + 8 + jbytes + 8;
  uint64_t len = off_tail + 8 + 12ull * nb_ + 8 + cap + 8 + 2ull * cap;
  uint32_t nch = (uint32_t)((len + 1023) / 1024);
  S.hbuf.ensure((size_t)nch * 1024 + 64);
  RP_CUDA(cudaMemsetAsync(S.hbuf.p, 0, (size_t)nch * 1024 + 64, st));
  uint8_t head[48];
  auto p64 = [&](uint8_t* p, uint64_t v) { for (int i = 0; i < 8; ++i) p[i] = (uint8_t)(v >> (8 * i)); };
  p64(head, epoch_);
  p64(head + 8, rng_);
  static const uint8_t kEmpty[32] = {0xaf, 0x13, 0x49, 0xb9, 0xf5, 0xf9, 0xa1, 0xa6, 0xa0, 0x40, 0x4d,
                                     0xea, 0x36, 0xdc, 0xc9, 0x49, 0x9b, 0xcb, 0x25, 0xc9, 0xad, 0xc1,
                                     0x12, 0xb7, 0xcc, 0x9a, 0x93, 0xca, 0xe4, 0x1f, 0x32, 0x62};
  std::memcpy(head + 16, kEmpty, 32);
  RP_CUDA(cudaMemcpyAsync(S.hbuf.p, head, 48, cudaMemcpyHostToDevice, st));
  if (nb_) { k_h_bodies<<<(nb_ + T - 1) / T, T, 0, st>>>(nb_, pos.p, rot.p, lin.p, ang.p, S.hbuf.p + off_bodies); RP_COUNT_LAUNCH(1); }
  uint8_t wcount[8];
  p64(wcount, nkeys);
  RP_CUDA(cudaMemcpyAsync(S.hbuf.p + off_warm, wcount, 8, cudaMemcpyHostToDevice, st));
  if (n_warm) {
    k_h_warm<<<(n_warm + T - 1) / T, T, 0, st>>>(n_warm, warm_key.p, warm_a.p, warm_b.p, S.woff.p, S.wpos.p,
                                                  S.hbuf.p + off_warm + 8); RP_COUNT_LAUNCH(1);
  }
  // the empty patch and rotor maps are zero bytes already; the joint section between them
  uint8_t jc[8];
  p64(jc, jcount);
  RP_CUDA(cudaMemcpyAsync(S.hbuf.p + off_joints, jc, 8, cudaMemcpyHostToDevice, st));
  joint_write(*this, 0, nj, S.jh_off.p, S.hbuf.p + off_joints + 8, st);
  uint32_t nt = cap > nb_ ? cap : nb_;
  k_h_tail<<<(nt + T) / T, T, 0, st>>>(nb_, cap, last_lin.p, awake.p, sleep_ticks.p, S.hbuf.p + off_tail); RP_COUNT_LAUNCH(1);
  S.hcv.ensure(16 * (size_t)nch + 16);
  uint32_t* root = S.hcv.p;
  uint32_t* a = S.hcv.p + 8;
  uint32_t* b = S.hcv.p + 8 + 8 * (size_t)nch;
  k_b3_chunks<<<(nch + 127) / 128, 128, 0, st>>>(S.hbuf.p, len, nch, a, root); RP_COUNT_LAUNCH(1);
  uint32_t n = nch;
  while (n > 1) {
    uint32_t n_out = (n + 1) / 2;
    k_b3_parents<<<(n_out + 127) / 128, 128, 0, st>>>(n, a, b, root); RP_COUNT_LAUNCH(1);
    std::swap(a, b);
    n = n_out;
  }
  uint32_t r[8];
  RP_CUDA(cudaMemcpyAsync(r, root, 32, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < 8; ++i)
    for (int k = 0; k < 4; ++k) out32[4 * i + k] = (uint8_t)(r[i] >> (8 * k));
}

// ------------------------------------------------------------------ one world of a batch
// The digest a World holding exactly world w's bodies would compute (capacity = its body count):
// bodies [b0, b1) with 0-based indices, the warm entries whose first body is in that range (one
// contiguous run of the sorted cache) with body ids made 0-based, and that range's carried state.
__global__ void k_warm_range(uint32_t n, const uint4* __restrict__ k, uint32_t b0, uint32_t b1, uint32_t* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t lo = 0, hi = n;
  while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (k[m].x < b0) lo = m + 1; else hi = m; }
  uint32_t a = lo;
  hi = n;
  while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (k[m].x < b1) lo = m + 1; else hi = m; }
  out[0] = a;
  out[1] = lo;
}
void WorldGpu::step_hash_world(uint32_t w, uint8_t out32[32]) {
  upload_joints();
  Scratch& S = *s_;
  cudaStream_t st = stream_;
  const int T = 256;
  uint32_t b0 = h_wb_start_[w], b1 = w + 1 < h_wb_start_.size() ? h_wb_start_[w + 1] : nb_;
  uint32_t nbw = b1 - b0, cap = nbw;
  uint32_t lohi[2] = {0, 0};
  S.counts.ensure(4);
  if (n_warm) {
    k_warm_range<<<1, 1, 0, st>>>(n_warm, warm_key.p, b0, b1, S.counts.p); RP_COUNT_LAUNCH(1);
    RP_CUDA(cudaMemcpyAsync(lohi, S.counts.p, 8, cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaStreamSynchronize(st));
  }
  uint32_t wlo = lohi[0], nw = lohi[1] - lohi[0];
  S.woff.ensure(nw + 1); S.wpos.ensure(nw + 1);
  uint32_t nkeys = 0;
  if (nw) {
    k_h_warm_flags<<<(nw + T - 1) / T, T, 0, st>>>(nw, warm_key.p + wlo, S.woff.p); RP_COUNT_LAUNCH(1);
    nkeys = exclusive_scan_total(S, S.woff.p, S.wpos.p, nw, st);
  }
  // the world's joints: one contiguous id range (a batch's joints join bodies of the world added last)
  uint32_t j0 = 0, j1 = 0;
  {
    auto first_at = [&](uint32_t b) {
      uint32_t lo = 0, hi = num_joints();
      while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (h_joints_[m].a < b) lo = m + 1; else hi = m; }
      return lo;
    };
    j0 = first_at(b0); j1 = first_at(b1);
  }
  const uint32_t njw = j1 - j0;
  uint64_t jbytes = 0, jcount = 0;
  S.jh_sz.ensure(njw + 1); S.jh_off.ensure(njw + 1); S.jh_has.ensure(njw + 1); S.jh_pos.ensure(njw + 1);
  joint_section(*this, j0, njw, S.jh_sz.p, S.jh_off.p, S.jh_has.p, S.jh_pos.p, &jbytes, &jcount, st);
  uint64_t off_bodies = 48;
  uint64_t off_warm = off_bodies + 56ull * nbw;
  uint64_t off_joints = off_warm + 8 + 20ull * nkeys + 28ull * nw + 8;
  uint64_t off_tail = off_joints + 8 + jbytes + 8;
  uint64_t len = off_tail + 8 + 12ull * nbw + 8 + cap + 8 + 2ull * cap;
  uint32_t nch = (uint32_t)((len + 1023) / 1024);
  S.hbuf.ensure((size_t)nch * 1024 + 64);
  RP_CUDA(cudaMemsetAsync(S.hbuf.p, 0, (size_t)nch * 1024 + 64, st));
  uint8_t head[48];
  auto p64 = [&](uint8_t* p, uint64_t v) { for (int i = 0; i < 8; ++i) p[i] = (uint8_t)(v >> (8 * i)); };
  p64(head, epoch_);
  p64(head + 8, rng_);
  static const uint8_t kEmpty[32] = {0xaf, 0x13, 0x49, 0xb9, 0xf5, 0xf9, 0xa1, 0xa6, 0xa0, 0x40, 0x4d,
                                     0xea, 0x36, 0xdc, 0xc9, 0x49, 0x9b, 0xcb, 0x25, 0xc9, 0xad, 0xc1,
                                     0x12, 0xb7, 0xcc, 0x9a, 0x93, 0xca, 0xe4, 0x1f, 0x32, 0x62};
  std::memcpy(head + 16, kEmpty, 32);
  uint8_t wcount[8];
  p64(wcount, nkeys);
  RP_CUDA(cudaMemcpyAsync(S.hbuf.p, head, 48, cudaMemcpyHostToDevice, st));
  if (nbw)
    k_h_bodies<<<(nbw + T - 1) / T, T, 0, st>>>(nbw, pos.p + b0, rot.p + b0, lin.p + b0, ang.p + b0, S.hbuf.p + off_bodies);
  if (nbw) RP_COUNT_LAUNCH(1);
  RP_CUDA(cudaMemcpyAsync(S.hbuf.p + off_warm, wcount, 8, cudaMemcpyHostToDevice, st));
  if (nw)
    k_h_warm<<<(nw + T - 1) / T, T, 0, st>>>(nw, warm_key.p + wlo, warm_a.p + wlo, warm_b.p + wlo, S.woff.p, S.wpos.p,
                                              S.hbuf.p + off_warm + 8, b0);
  if (nw) RP_COUNT_LAUNCH(1);
  uint8_t jc[8];
  p64(jc, jcount);
  RP_CUDA(cudaMemcpyAsync(S.hbuf.p + off_joints, jc, 8, cudaMemcpyHostToDevice, st));
  joint_write(*this, j0, njw, S.jh_off.p, S.hbuf.p + off_joints + 8, st);
  k_h_tail<<<(nbw + T) / T, T, 0, st>>>(nbw, cap, last_lin.p + b0, awake.p + b0, sleep_ticks.p + b0, S.hbuf.p + off_tail);
  RP_COUNT_LAUNCH(1);
  S.hcv.ensure(16 * (size_t)nch + 16);
  uint32_t* root = S.hcv.p;
  uint32_t* a = S.hcv.p + 8;
  uint32_t* b = S.hcv.p + 8 + 8 * (size_t)nch;
  k_b3_chunks<<<(nch + 127) / 128, 128, 0, st>>>(S.hbuf.p, len, nch, a, root); RP_COUNT_LAUNCH(1);
  uint32_t n = nch;
  while (n > 1) {
    uint32_t n_out = (n + 1) / 2;
    k_b3_parents<<<(n_out + 127) / 128, 128, 0, st>>>(n, a, b, root); RP_COUNT_LAUNCH(1);
    std::swap(a, b);
    n = n_out;
  }
  uint32_t r[8];
  RP_CUDA(cudaMemcpyAsync(r, root, 32, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < 8; ++i)
    for (int k = 0; k < 4; ++k) out32[4 * i + k] = (uint8_t)(r[i] >> (8 * k));
}

// ------------------------------------------------------------------ allocation-free variant
// step_hash_noalloc writes the same stream and runs the same kernels as step_hash, but every
// scratch byte lives in g_noalloc_scratch, a fixed array in device memory reserved when the library
// is loaded: no cudaMalloc / cudaFree and no allocating library routine on any call. Layout:
//   [stream: NOALLOC_STREAM_MAX + 1088 B][chaining values: 16 * (NOALLOC_STREAM_MAX / 1024 + 1) + 16
//   words][warm key starts: NOALLOC_WARM_MAX + 1 words][warm key ranks: same][joint entry sizes,
//   offsets, flags, ranks: NOALLOC_JOINT_MAX + 1 words each][scan temp: 64 KiB].
// Only the stream must start at zero; each call clears the part it uses. The array is one per
// device and shared by every world on it: two calls in flight at once would overwrite each other's
// bytes, so calls are serialised by g_noalloc_mu and each returns after its work on the device ended.
#define NOALLOC_STREAM_MAX (12u << 20)   // bytes of serialised state (about 150k bodies, few warm entries)
#define NOALLOC_WARM_MAX (256u << 10)    // warm-start entries
#define NOALLOC_CHUNKS (NOALLOC_STREAM_MAX / 1024u + 1u)
#define NOALLOC_OFF_CV ((size_t)NOALLOC_STREAM_MAX + 1088u)
#define NOALLOC_OFF_WOFF (NOALLOC_OFF_CV + 4u * (16u * (size_t)NOALLOC_CHUNKS + 16u))
#define NOALLOC_OFF_WPOS (NOALLOC_OFF_WOFF + 4u * ((size_t)NOALLOC_WARM_MAX + 1u))
#define NOALLOC_JOINT_MAX (64u << 10)    // joints
#define NOALLOC_OFF_JSZ (NOALLOC_OFF_WPOS + 4u * ((size_t)NOALLOC_WARM_MAX + 1u))
#define NOALLOC_OFF_JOFF (NOALLOC_OFF_JSZ + 4u * ((size_t)NOALLOC_JOINT_MAX + 1u))
#define NOALLOC_OFF_JHAS (NOALLOC_OFF_JOFF + 4u * ((size_t)NOALLOC_JOINT_MAX + 1u))
#define NOALLOC_OFF_JPOS (NOALLOC_OFF_JHAS + 4u * ((size_t)NOALLOC_JOINT_MAX + 1u))
#define NOALLOC_OFF_TEMP ((NOALLOC_OFF_JPOS + 4u * ((size_t)NOALLOC_JOINT_MAX + 1u) + 255u) & ~(size_t)255u)
#define NOALLOC_TEMP_BYTES (64u << 10)
#define NOALLOC_BYTES (NOALLOC_OFF_TEMP + NOALLOC_TEMP_BYTES)
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_ptr[64];  // per device ordinal, set by the first call on that device

// The device address of g_noalloc_scratch on device dev (the current device), looked up on the
// first call there.
static unsigned char* noalloc_scratch(int dev) {
  if (dev < 0 || dev >= 64) throw std::runtime_error("step_hash_noalloc: device ordinal above 63");
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    RP_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
  }
  return g_noalloc_ptr[dev];
}
// Makes the world's device current for the call and puts the caller's back on return.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    RP_CUDA(cudaGetDevice(&prev));
    if (prev != dev) RP_CUDA(cudaSetDevice(dev));
    else prev = -1;
  }
  ~DeviceScope() { if (prev >= 0) cudaSetDevice(prev); }
};

void WorldGpu::step_hash_noalloc(uint8_t out32[32]) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  const int T = 256;
  uint32_t cap = cap_b_ > nb_ ? cap_b_ : nb_;
  // Every limit is checked before any device work. Joints added or changed since the last tick
  // are not uploaded here (that would allocate): the warm cache holds entries for the first
  // jw_init_ joints only, and a joint without an entry adds no byte to the stream, so hashing
  // those jw_init_ slots gives the digest step_hash gives after its upload.
  if (num_joints() > NOALLOC_JOINT_MAX)
    throw std::length_error("step_hash_noalloc: " + std::to_string(num_joints()) + " joints, at most " +
                            std::to_string(NOALLOC_JOINT_MAX));
  if (n_warm > NOALLOC_WARM_MAX)
    throw std::length_error("step_hash_noalloc: " + std::to_string(n_warm) + " warm-start entries, at most " +
                            std::to_string(NOALLOC_WARM_MAX));
  const uint32_t nj = jw_n.p ? jw_init_ : 0u;
  // the stream length bound holds with every warm entry under its own key (the most bytes) and
  // every joint holding the most rows
  uint64_t worst = 48 + 56ull * nb_ + 8 + 48ull * n_warm + 24 + (8 + 5ull * kJointRows) * nj + 8 + 12ull * nb_ + 8 + cap + 8 +
                   2ull * cap;
  if (worst > NOALLOC_STREAM_MAX)
    throw std::length_error("step_hash_noalloc: state stream of up to " + std::to_string(worst) + " bytes (" +
                            std::to_string(nb_) + " bodies, capacity " + std::to_string(cap) + ", " +
                            std::to_string(n_warm) + " warm entries), at most " + std::to_string(NOALLOC_STREAM_MAX));
  // the scans' temporary bytes (cub's size query launches nothing)
  size_t wtemp = 0, jtemp = 0;
  if (n_warm) RP_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, wtemp, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)n_warm, stream_));
  if (nj) RP_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, jtemp, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)nj, stream_));
  if (wtemp > NOALLOC_TEMP_BYTES || jtemp > NOALLOC_TEMP_BYTES)
    throw std::length_error("step_hash_noalloc: scan needs more temporary bytes than reserved");
  DeviceScope on_device(dev_);
  unsigned char* base = noalloc_scratch(dev_);
  cudaStream_t st = stream_;
  uint32_t* woff = reinterpret_cast<uint32_t*>(base + NOALLOC_OFF_WOFF);
  uint32_t* wpos = reinterpret_cast<uint32_t*>(base + NOALLOC_OFF_WPOS);
  uint32_t* jsz = reinterpret_cast<uint32_t*>(base + NOALLOC_OFF_JSZ);
  uint32_t* joff = reinterpret_cast<uint32_t*>(base + NOALLOC_OFF_JOFF);
  uint32_t* jhas = reinterpret_cast<uint32_t*>(base + NOALLOC_OFF_JHAS);
  uint32_t* jpos = reinterpret_cast<uint32_t*>(base + NOALLOC_OFF_JPOS);
  void* temp = base + NOALLOC_OFF_TEMP;
  uint32_t nkeys = 0;
  if (n_warm) {
    size_t bytes = wtemp;
    k_h_warm_flags<<<(n_warm + T - 1) / T, T, 0, st>>>(n_warm, warm_key.p, woff); RP_COUNT_LAUNCH(1);
    RP_CUDA(cub::DeviceScan::ExclusiveSum(temp, bytes, woff, wpos, (int)n_warm, st));
    RP_COUNT_LAUNCH(2);
    uint32_t a = 0, b = 0;
    RP_CUDA(cudaMemcpyAsync(&a, wpos + n_warm - 1, 4, cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaMemcpyAsync(&b, woff + n_warm - 1, 4, cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaStreamSynchronize(st));
    nkeys = a + b;
  }
  uint64_t jbytes = 0, jcount = 0;
  if (nj) {
    size_t bytes = jtemp;
    k_hj_sizes<<<(nj + T - 1) / T, T, 0, st>>>(nj, jw_n.p, jsz, jhas); RP_COUNT_LAUNCH(1);
    RP_CUDA(cub::DeviceScan::ExclusiveSum(temp, bytes, jsz, joff, (int)nj, st));
    RP_COUNT_LAUNCH(2);
    RP_CUDA(cub::DeviceScan::ExclusiveSum(temp, bytes, jhas, jpos, (int)nj, st));
    RP_COUNT_LAUNCH(2);
    uint32_t v[4] = {0, 0, 0, 0};
    RP_CUDA(cudaMemcpyAsync(&v[0], joff + nj - 1, 4, cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaMemcpyAsync(&v[1], jsz + nj - 1, 4, cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaMemcpyAsync(&v[2], jpos + nj - 1, 4, cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaMemcpyAsync(&v[3], jhas + nj - 1, 4, cudaMemcpyDeviceToHost, st));
    RP_CUDA(cudaStreamSynchronize(st));
    jbytes = (uint64_t)v[0] + v[1];
    jcount = (uint64_t)v[2] + v[3];
  }
  uint64_t off_bodies = 48;
  uint64_t off_warm = off_bodies + 56ull * nb_;
  uint64_t off_joints = off_warm + 8 + 20ull * nkeys + 28ull * n_warm + 8;
  uint64_t off_tail = off_joints + 8 + jbytes + 8;
  uint64_t len = off_tail + 8 + 12ull * nb_ + 8 + cap + 8 + 2ull * cap;
  uint32_t nch = (uint32_t)((len + 1023) / 1024);
  uint8_t* hbuf = base;
  RP_CUDA(cudaMemsetAsync(hbuf, 0, (size_t)nch * 1024 + 64, st));
  uint8_t head[48];
  auto p64 = [&](uint8_t* p, uint64_t v) { for (int i = 0; i < 8; ++i) p[i] = (uint8_t)(v >> (8 * i)); };
  p64(head, epoch_);
  p64(head + 8, rng_);
  static const uint8_t kEmpty[32] = {0xaf, 0x13, 0x49, 0xb9, 0xf5, 0xf9, 0xa1, 0xa6, 0xa0, 0x40, 0x4d,
                                     0xea, 0x36, 0xdc, 0xc9, 0x49, 0x9b, 0xcb, 0x25, 0xc9, 0xad, 0xc1,
                                     0x12, 0xb7, 0xcc, 0x9a, 0x93, 0xca, 0xe4, 0x1f, 0x32, 0x62};
  std::memcpy(head + 16, kEmpty, 32);
  uint8_t wcount[8];
  p64(wcount, nkeys);
  RP_CUDA(cudaMemcpyAsync(hbuf, head, 48, cudaMemcpyHostToDevice, st));
  if (nb_) { k_h_bodies<<<(nb_ + T - 1) / T, T, 0, st>>>(nb_, pos.p, rot.p, lin.p, ang.p, hbuf + off_bodies); RP_COUNT_LAUNCH(1); }
  RP_CUDA(cudaMemcpyAsync(hbuf + off_warm, wcount, 8, cudaMemcpyHostToDevice, st));
  if (n_warm)
    k_h_warm<<<(n_warm + T - 1) / T, T, 0, st>>>(n_warm, warm_key.p, warm_a.p, warm_b.p, woff, wpos, hbuf + off_warm + 8);
  if (n_warm) RP_COUNT_LAUNCH(1);
  uint8_t jc[8];
  p64(jc, jcount);
  RP_CUDA(cudaMemcpyAsync(hbuf + off_joints, jc, 8, cudaMemcpyHostToDevice, st));
  joint_write(*this, 0, nj, joff, hbuf + off_joints + 8, st);
  uint32_t nt = cap > nb_ ? cap : nb_;
  k_h_tail<<<(nt + T) / T, T, 0, st>>>(nb_, cap, last_lin.p, awake.p, sleep_ticks.p, hbuf + off_tail); RP_COUNT_LAUNCH(1);
  uint32_t* cv = reinterpret_cast<uint32_t*>(base + NOALLOC_OFF_CV);
  uint32_t* root = cv;
  uint32_t* a = cv + 8;
  uint32_t* b = cv + 8 + 8 * (size_t)nch;
  k_b3_chunks<<<(nch + 127) / 128, 128, 0, st>>>(hbuf, len, nch, a, root); RP_COUNT_LAUNCH(1);
  uint32_t n = nch;
  while (n > 1) {
    uint32_t n_out = (n + 1) / 2;
    k_b3_parents<<<(n_out + 127) / 128, 128, 0, st>>>(n, a, b, root); RP_COUNT_LAUNCH(1);
    std::swap(a, b);
    n = n_out;
  }
  uint32_t r[8];
  RP_CUDA(cudaMemcpyAsync(r, root, 32, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < 8; ++i)
    for (int k = 0; k < 4; ++k) out32[4 * i + k] = (uint8_t)(r[i] >> (8 * k));
}

}  // namespace rp

namespace rp {
// ------------------------------------------------------------------ every world of a batch at once
// The digests step_hash_world gives, for worlds [first, first + count), from kernels that walk the
// world table: per world its body range, warm-cache range (binary search on the sorted keys), key
// and joint-entry counts (differences of prefix sums over the whole cache), stream length and
// chunk count (k_wh_meta); then, per slice of worlds whose streams fit the scratch, every world's
// stream written at its chunk offset by one thread per record, one thread per 1 KiB chunk over all
// the slice's worlds (k_wh_chunks), and one block per world merging its parent tree (k_wh_tree).
struct WhMeta {
  uint32_t b0, nb, wlo, nw, g0, nkeys, j0, njw, jo0, jbytes, jcount, nch;
  unsigned long long len;
};
__global__ void k_wh_meta(uint32_t nwld, uint32_t w0, const uint32_t* __restrict__ wbs, uint32_t nb_total,
                          const uint4* __restrict__ wk, uint32_t n_warm, const uint32_t* __restrict__ gflag,
                          const uint32_t* __restrict__ gpre, const uint32_t* __restrict__ jrange,
                          const uint32_t* __restrict__ jsz, const uint32_t* __restrict__ joff,
                          const uint32_t* __restrict__ jhas, const uint32_t* __restrict__ jpos, WhMeta* meta) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nwld) return;
  uint32_t w = w0 + k;
  WhMeta m;
  m.b0 = wbs[w];
  uint32_t b1 = wbs[w + 1] < nb_total ? wbs[w + 1] : nb_total;
  m.nb = b1 - m.b0;
  auto lower = [&](uint32_t b) {
    uint32_t lo = 0, hi = n_warm;
    while (lo < hi) { uint32_t md = (lo + hi) >> 1; if (wk[md].x < b) lo = md + 1; else hi = md; }
    return lo;
  };
  m.wlo = lower(m.b0);
  uint32_t whi = lower(b1);
  m.nw = whi - m.wlo;
  m.g0 = m.nw ? gpre[m.wlo] : 0u;
  m.nkeys = m.nw ? (gpre[whi - 1] + gflag[whi - 1]) - gpre[m.wlo] : 0u;
  m.j0 = jrange[2 * w];
  m.njw = jrange[2 * w + 1] - m.j0;
  m.jo0 = m.njw ? joff[m.j0] : 0u;
  m.jbytes = m.njw ? (joff[m.j0 + m.njw - 1] + jsz[m.j0 + m.njw - 1]) - m.jo0 : 0u;
  m.jcount = m.njw ? (jpos[m.j0 + m.njw - 1] + jhas[m.j0 + m.njw - 1]) - jpos[m.j0] : 0u;
  const unsigned long long cap = m.nb;
  m.len = 48ull + 56ull * m.nb + 8 + 20ull * m.nkeys + 28ull * m.nw + 8 + 8 + m.jbytes + 8 + 8 + 12ull * m.nb + 8 + cap +
          8 + 2ull * cap;
  m.nch = (uint32_t)((m.len + 1023) / 1024);
  meta[w] = m;
}
__device__ __forceinline__ uint32_t wh_world_of(const unsigned long long* __restrict__ ch0, uint32_t lo, uint32_t hi,
                                                unsigned long long c) {  // last world of [lo, hi) starting at or before c
  while (hi - lo > 1) { uint32_t md = (lo + hi) >> 1; if (ch0[md] <= c) lo = md; else hi = md; }
  return lo;
}
// the fixed parts of every world's stream: header, section counts
__global__ void k_wh_head(uint32_t w0, uint32_t nwld, const WhMeta* __restrict__ meta,
                          const unsigned long long* __restrict__ ch0, unsigned long long epoch, unsigned long long rng,
                          uint8_t* buf) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nwld) return;
  const WhMeta m = meta[w0 + k];
  uint8_t* p = buf + (ch0[k] - ch0[0]) * 1024ull;
  const uint8_t empty[32] = {0xaf, 0x13, 0x49, 0xb9, 0xf5, 0xf9, 0xa1, 0xa6, 0xa0, 0x40, 0x4d, 0xea, 0x36, 0xdc, 0xc9, 0x49,
                             0x9b, 0xcb, 0x25, 0xc9, 0xad, 0xc1, 0x12, 0xb7, 0xcc, 0x9a, 0x93, 0xca, 0xe4, 0x1f, 0x32, 0x62};
  put64(p, epoch);
  put64(p + 8, rng);
  for (int i = 0; i < 32; ++i) p[16 + i] = empty[i];
  const unsigned long long off_warm = 48ull + 56ull * m.nb;
  put64(p + off_warm, m.nkeys);
  const unsigned long long off_joints = off_warm + 8 + 20ull * m.nkeys + 28ull * m.nw + 8;
  put64(p + off_joints, m.jcount);
}
// body records and the carried tail of each world (0-based ids; capacity = the world's body count)
__global__ void k_wh_bodies(uint32_t w0, uint32_t nwld, uint32_t bfirst, uint32_t nbod, const uint32_t* __restrict__ wbs,
                            const WhMeta* __restrict__ meta, const unsigned long long* __restrict__ ch0,
                            const float4* __restrict__ pos, const float4* __restrict__ rot, const float4* __restrict__ lin,
                            const float4* __restrict__ ang, const float4* __restrict__ last,
                            const uint8_t* __restrict__ awake, const uint16_t* __restrict__ ticks, uint8_t* buf) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nbod) return;
  const uint32_t i = bfirst + t;
  uint32_t lo = 0, hi = nwld;  // the world holding body i
  while (hi - lo > 1) { uint32_t md = (lo + hi) >> 1; if (wbs[w0 + md] <= i) lo = md; else hi = md; }
  const WhMeta m = meta[w0 + lo];
  uint8_t* s = buf + (ch0[lo] - ch0[0]) * 1024ull;
  const uint32_t li = i - m.b0;
  uint8_t* p = s + 48 + 56ull * li;
  float4 a = pos[i], q = rot[i], l = lin[i], w = ang[i];
  put32(p, li);
  put32(p + 4, canon_bits(a.x)); put32(p + 8, canon_bits(a.y)); put32(p + 12, canon_bits(a.z));
  put32(p + 16, canon_bits(q.x)); put32(p + 20, canon_bits(q.y)); put32(p + 24, canon_bits(q.z)); put32(p + 28, canon_bits(q.w));
  put32(p + 32, canon_bits(l.x)); put32(p + 36, canon_bits(l.y)); put32(p + 40, canon_bits(l.z));
  put32(p + 44, canon_bits(w.x)); put32(p + 48, canon_bits(w.y)); put32(p + 52, canon_bits(w.z));
  // tail: [u64 nb][12 nb][u64 cap][cap][u64 cap][2 cap]
  uint8_t* tl = s + 48ull + 56ull * m.nb + 8 + 20ull * m.nkeys + 28ull * m.nw + 8 + 8 + m.jbytes + 8;
  if (li == 0) put64(tl, m.nb);
  float4 v = last[i];
  put32(tl + 8 + 12ull * li, canon_bits(v.x)); put32(tl + 12 + 12ull * li, canon_bits(v.y));
  put32(tl + 16 + 12ull * li, canon_bits(v.z));
  uint8_t* aw = tl + 8 + 12ull * m.nb;
  if (li == 0) put64(aw, m.nb);
  aw[8 + li] = awake[i];
  uint8_t* tk = aw + 8 + m.nb;
  if (li == 0) put64(tk, m.nb);
  uint16_t tv = ticks[i];
  tk[8 + 2 * li] = (uint8_t)tv;
  tk[9 + 2 * li] = (uint8_t)(tv >> 8);
}
// warm-cache entries [efirst, efirst + n) of the slice: key headers and entries, ids 0-based
__global__ void k_wh_warm(uint32_t w0, uint32_t nwld, uint32_t efirst, uint32_t n, const uint32_t* __restrict__ wbs,
                          const WhMeta* __restrict__ meta, const unsigned long long* __restrict__ ch0,
                          const uint4* __restrict__ wk, const float4* __restrict__ wa, const float4* __restrict__ wb,
                          const uint32_t* __restrict__ gflag, const uint32_t* __restrict__ gpre, uint32_t n_warm, uint8_t* buf) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t e = efirst + t;
  const uint4 key = wk[e];
  uint32_t lo = 0, hi = nwld;  // the world of the key's first body
  while (hi - lo > 1) { uint32_t md = (lo + hi) >> 1; if (wbs[w0 + md] <= key.x) lo = md; else hi = md; }
  const WhMeta m = meta[w0 + lo];
  uint8_t* out = buf + (ch0[lo] - ch0[0]) * 1024ull + 48ull + 56ull * m.nb + 8;
  const uint32_t le = e - m.wlo, g = gpre[e] + gflag[e] - 1 - m.g0;
  if (gflag[e]) {
    uint32_t cnt = 1;
    while (e + cnt < n_warm && !gflag[e + cnt]) cnt++;
    uint8_t* h = out + 20ull * g + 28ull * le;
    put32(h, key.x - m.b0); put32(h + 4, key.y == 0xFFFFFFFFu ? key.y : key.y - m.b0);
    put32(h + 8, key.z); put32(h + 12, key.w); put32(h + 16, cnt);
  }
  uint8_t* p = out + 20ull * (g + 1) + 28ull * le;
  float4 a = wa[e], b = wb[e];
  put32(p, canon_bits(a.x)); put32(p + 4, canon_bits(a.y)); put32(p + 8, canon_bits(a.z)); put32(p + 12, canon_bits(a.w));
  put32(p + 16, canon_bits(b.x)); put32(p + 20, canon_bits(b.y)); put32(p + 24, canon_bits(b.z));
}
// joint-cache entries of joints [jfirst, jfirst + n) of the slice, joint ids 0-based per world
__global__ void k_wh_joints(uint32_t w0, uint32_t nwld, uint32_t jfirst, uint32_t n, const uint32_t* __restrict__ jrange,
                            const WhMeta* __restrict__ meta, const unsigned long long* __restrict__ ch0,
                            const uint32_t* __restrict__ jw_n,
                            const uint8_t* __restrict__ tag, const float* __restrict__ lam,
                            const uint32_t* __restrict__ joff, uint8_t* buf) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t j = jfirst + t;
  const uint32_t c = jw_n[j];
  if (c == 0xFFFFFFFFu) return;
  uint32_t lo = 0, hi = nwld;  // the last world whose joint range starts at or before j (empty ones come first)
  while (hi - lo > 1) { uint32_t md = (lo + hi) >> 1; if (jrange[2 * (w0 + md)] <= j) lo = md; else hi = md; }
  const WhMeta m = meta[w0 + lo];
  uint8_t* p = buf + (ch0[lo] - ch0[0]) * 1024ull + 48ull + 56ull * m.nb + 8 + 20ull * m.nkeys + 28ull * m.nw + 8 + 8 +
               (joff[j] - m.jo0);
  put32(p, j - m.j0);
  put32(p + 4, c);
  for (uint32_t k = 0; k < c; ++k) {
    p[8 + 5 * k] = tag[kJointRows * (size_t)j + k];
    put32(p + 9 + 5 * k, canon_bits(lam[kJointRows * (size_t)j + k]));
  }
}
// one thread per 1 KiB chunk of the slice's streams: chaining values, or the root of a one-chunk world
__global__ void k_wh_chunks(uint32_t w0, uint32_t nwld, unsigned long long nchunks, const WhMeta* __restrict__ meta,
                            const unsigned long long* __restrict__ ch0, const uint8_t* __restrict__ buf, uint32_t* cvs,
                            uint32_t* roots) {
  unsigned long long gc = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gc >= nchunks) return;
  const unsigned long long c_abs = ch0[0] + gc;
  const uint32_t k = wh_world_of(ch0, 0, nwld, c_abs);
  const WhMeta m = meta[w0 + k];
  const unsigned long long c = c_abs - ch0[k];
  const unsigned long long base = c * 1024ull;
  const unsigned long long clen = m.len - base < 1024ull ? m.len - base : 1024ull;
  const uint32_t nblocks = clen == 0 ? 1u : (uint32_t)((clen + 63) / 64);
  const uint8_t* data = buf + (ch0[k] - ch0[0]) * 1024ull + base;
  uint32_t cv[8];
  for (int i = 0; i < 8; ++i) cv[i] = c_iv[i];
  for (uint32_t b = 0; b < nblocks; ++b) {
    uint32_t blk[16];
    const uint32_t* wds = reinterpret_cast<const uint32_t*>(data + 64ull * b);
    for (int i = 0; i < 16; ++i) blk[i] = wds[i];
    uint32_t blen = b + 1 == nblocks ? (uint32_t)(clen - 64ull * b) : 64u;
    uint32_t flags = (b == 0 ? CHUNK_START : 0u) | (b + 1 == nblocks ? CHUNK_END : 0u);
    if (m.nch == 1 && b + 1 == nblocks) flags |= ROOT;
    uint32_t o[8];
    b3_compress(cv, blk, c, blen, flags, o);
    for (int i = 0; i < 8; ++i) cv[i] = o[i];
  }
  uint32_t* dst = m.nch == 1 ? roots + 8ull * k : cvs + 8ull * (c_abs - ch0[0]);
  for (int i = 0; i < 8; ++i) dst[i] = cv[i];
}
// one block per world of the slice: its parent tree, level by level (left-complete: an odd last
// node moves up unchanged), ping-ponging between the chunk values and a second buffer
__global__ void k_wh_tree(uint32_t w0, const WhMeta* __restrict__ meta, const unsigned long long* __restrict__ ch0,
                          uint32_t* cvs, uint32_t* cvs2, uint32_t* roots) {
  const uint32_t k = blockIdx.x;
  const WhMeta m = meta[w0 + k];
  if (m.nch <= 1) return;
  uint32_t* a = cvs + 8ull * (ch0[k] - ch0[0]);
  uint32_t* b = cvs2 + 8ull * (ch0[k] - ch0[0]);
  uint32_t n = m.nch;
  while (n > 1) {
    const uint32_t n_out = (n + 1) / 2;
    for (uint32_t t = threadIdx.x; t < n_out; t += blockDim.x) {
      if (2 * t + 1 < n) {
        uint32_t blk[16], cv[8], o[8];
        for (int i = 0; i < 8; ++i) { blk[i] = a[16 * t + i]; blk[8 + i] = a[16 * t + 8 + i]; cv[i] = c_iv[i]; }
        b3_compress(cv, blk, 0, 64, PARENT | (n == 2 ? ROOT : 0u), o);
        uint32_t* dst = n == 2 ? roots + 8ull * k : b + 8 * t;
        for (int i = 0; i < 8; ++i) dst[i] = o[i];
      } else {
        for (int i = 0; i < 8; ++i) b[8 * t + i] = a[16 * t + i];
      }
    }
    __syncthreads();
    uint32_t* tmp = a; a = b; b = tmp;
    n = n_out;
  }
}

void WorldGpu::step_hash_worlds(uint32_t first, uint32_t count, uint8_t* out) {
  if (!count) return;
  upload_joints();
  upload_worlds();
  Scratch& S = *s_;
  cudaStream_t st = stream_;
  const int T = 256;
  const uint32_t nwt = num_worlds(), nj = num_joints();
  // the world table (body starts + end) and each world's joint id range, from the host mirrors
  std::vector<uint32_t> wbs(nwt + 1), jr(2 * (size_t)nwt);
  for (uint32_t w = 0; w < nwt; ++w) wbs[w] = h_wb_start_[w];
  wbs[nwt] = nb_;
  auto first_at = [&](uint32_t b) {
    uint32_t lo = 0, hi = nj;
    while (lo < hi) { uint32_t m = (lo + hi) >> 1; if (h_joints_[m].a < b) lo = m + 1; else hi = m; }
    return lo;
  };
  for (uint32_t w = 0; w < nwt; ++w) { jr[2 * w] = first_at(wbs[w]); jr[2 * w + 1] = first_at(wbs[w + 1]); }
  static_assert(sizeof(WhMeta) == 56, "WhMeta: 7 eight-byte words");
  S.wh_wbs.ensure(nwt + 1); S.wh_jr.ensure(2 * (size_t)nwt + 2); S.wh_meta.ensure(7 * (size_t)nwt + 7);
  RP_CUDA(cudaMemcpyAsync(S.wh_wbs.p, wbs.data(), 4 * wbs.size(), cudaMemcpyHostToDevice, st));
  RP_CUDA(cudaMemcpyAsync(S.wh_jr.p, jr.data(), 4 * jr.size(), cudaMemcpyHostToDevice, st));
  // key groups of the whole warm cache and the joint entries' sizes, as prefix sums
  S.woff.ensure(n_warm + 1); S.wpos.ensure(n_warm + 1);
  if (n_warm) {
    k_h_warm_flags<<<(n_warm + T - 1) / T, T, 0, st>>>(n_warm, warm_key.p, S.woff.p); RP_COUNT_LAUNCH(1);
    exclusive_scan_total(S, S.woff.p, S.wpos.p, n_warm, st);
  }
  S.jh_sz.ensure(nj + 1); S.jh_off.ensure(nj + 1); S.jh_has.ensure(nj + 1); S.jh_pos.ensure(nj + 1);
  if (nj) {
    k_hj_sizes<<<(nj + T - 1) / T, T, 0, st>>>(nj, jw_n.p, S.jh_sz.p, S.jh_has.p); RP_COUNT_LAUNCH(1);
    exclusive_scan_total(S, S.jh_sz.p, S.jh_off.p, nj, st);
    exclusive_scan_total(S, S.jh_has.p, S.jh_pos.p, nj, st);
  }
  WhMeta* meta = reinterpret_cast<WhMeta*>(S.wh_meta.p);
  k_wh_meta<<<(count + T - 1) / T, T, 0, st>>>(count, first, S.wh_wbs.p, nb_, warm_key.p, n_warm, S.woff.p, S.wpos.p,
                                                S.wh_jr.p, S.jh_sz.p, S.jh_off.p, S.jh_has.p, S.jh_pos.p, meta);
  RP_COUNT_LAUNCH(1);
  std::vector<WhMeta> hm(count);
  RP_CUDA(cudaMemcpyAsync(hm.data(), meta + first, sizeof(WhMeta) * count, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
  // slices of worlds whose streams fit 64 MiB (a world larger than that is a slice alone)
  const unsigned long long budget = 64ull << 10;  // chunks
  S.wh_roots.ensure(8 * (size_t)count + 8);
  uint32_t w = 0;
  while (w < count) {
    uint32_t e = w;
    unsigned long long chunks = 0;
    std::vector<unsigned long long> ch0;
    while (e < count && (e == w || chunks + hm[e].nch <= budget)) { ch0.push_back(chunks); chunks += hm[e].nch; e++; }
    const uint32_t nwl = e - w;
    ch0.push_back(chunks);
    S.wh_ch0.ensure(ch0.size());
    S.hbuf.ensure((size_t)chunks * 1024 + 64);
    S.hcv.ensure(16 * (size_t)chunks + 16);
    RP_CUDA(cudaMemcpyAsync(S.wh_ch0.p, ch0.data(), 8 * ch0.size(), cudaMemcpyHostToDevice, st));
    RP_CUDA(cudaMemsetAsync(S.hbuf.p, 0, (size_t)chunks * 1024 + 64, st));
    const uint32_t wg = first + w;
    k_wh_head<<<(nwl + T - 1) / T, T, 0, st>>>(wg, nwl, meta, S.wh_ch0.p, epoch_, rng_, S.hbuf.p); RP_COUNT_LAUNCH(1);
    const uint32_t bfirst = hm[w].b0, nbod = hm[e - 1].b0 + hm[e - 1].nb - bfirst;
    if (nbod) {
      k_wh_bodies<<<(nbod + T - 1) / T, T, 0, st>>>(wg, nwl, bfirst, nbod, S.wh_wbs.p, meta, S.wh_ch0.p, pos.p, rot.p, lin.p,
                                                    ang.p, last_lin.p, awake.p, sleep_ticks.p, S.hbuf.p);
      RP_COUNT_LAUNCH(1);
    }
    const uint32_t efirst = hm[w].wlo, nent = hm[e - 1].wlo + hm[e - 1].nw - efirst;
    if (nent) {
      k_wh_warm<<<(nent + T - 1) / T, T, 0, st>>>(wg, nwl, efirst, nent, S.wh_wbs.p, meta, S.wh_ch0.p, warm_key.p, warm_a.p,
                                                  warm_b.p, S.woff.p, S.wpos.p, n_warm, S.hbuf.p);
      RP_COUNT_LAUNCH(1);
    }
    const uint32_t jfirst = hm[w].j0, njs = hm[e - 1].j0 + hm[e - 1].njw - jfirst;
    if (njs) {
      k_wh_joints<<<(njs + T - 1) / T, T, 0, st>>>(wg, nwl, jfirst, njs, S.wh_jr.p, meta, S.wh_ch0.p, jw_n.p,
                                                   jw_tag.p, jw_lam.p, S.jh_off.p, S.hbuf.p);
      RP_COUNT_LAUNCH(1);
    }
    k_wh_chunks<<<(unsigned)((chunks + 127) / 128), 128, 0, st>>>(wg, nwl, chunks, meta, S.wh_ch0.p, S.hbuf.p, S.hcv.p,
                                                                  S.wh_roots.p + 8ull * w);
    RP_COUNT_LAUNCH(1);
    k_wh_tree<<<nwl, 128, 0, st>>>(wg, meta, S.wh_ch0.p, S.hcv.p, S.hcv.p + 8 * (size_t)chunks + 8, S.wh_roots.p + 8ull * w);
    RP_COUNT_LAUNCH(1);
    w = e;
  }
  std::vector<uint32_t> r(8 * (size_t)count);
  RP_CUDA(cudaMemcpyAsync(r.data(), S.wh_roots.p, 32 * (size_t)count, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
  for (uint32_t k = 0; k < count; ++k)
    for (int i = 0; i < 8; ++i)
      for (int b = 0; b < 4; ++b) out[32 * (size_t)k + 4 * i + b] = (uint8_t)(r[8 * (size_t)k + i] >> (8 * b));
}
}  // namespace rp
