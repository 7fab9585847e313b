// wire.cu -- the riftnet snapshot packed on the device (riftphys-riftnet/src/wire.rs:1-53): every
// live body as a NetEnt (id, pose, scale, kind), 25 to a chunk behind a NetHdr, the chunks back to
// back, ready for a host to send one datagram per chunk. One thread per body writes its 48 bytes,
// one per chunk its 32-byte header; the only host work is the copy of the result.
#include <cstring>

#include "step_internal.cuh"

namespace rp {

namespace {
const int T = 256;
inline int nblk(uint32_t n, int t = T) { return n ? (int)((n + t - 1) / t) : 1; }
}  // namespace

// wire.rs:4-6, 35
constexpr uint32_t kWireMagic = 0x30535052u;
constexpr uint32_t kWireVer = 2u, kWireKindSnapshot = 1u;
constexpr uint32_t kWireHdr = 32u, kWireEnt = 48u, kWirePer = 1200u / 48u;  // MAX_PAYLOAD / size_of::<NetEnt>()
constexpr uint32_t kWireChunk = kWireHdr + kWirePer * kWireEnt;

__global__ void k_wire_flags(uint32_t nb, const uint8_t* __restrict__ alive, uint32_t* flag) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) flag[i] = alive[i] ? 1u : 0u;
}
// NetEnt (wire.rs:24-33): kind 1 sphere, 2 box, 3 capsule along y, scale (r, r, r), the half
// extents, or (r, (hh + r) / 2, r).
__global__ void k_wire_ents(uint32_t nb, const uint8_t* __restrict__ alive, const uint32_t* __restrict__ off,
                            const float4* __restrict__ pos, const float4* __restrict__ rot,
                            const uint32_t* __restrict__ col_kind, const float4* __restrict__ col_dims, uint8_t* out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb || !alive[i]) return;
  const uint32_t e = off[i], c = e / kWirePer, s = e % kWirePer;
  float4* dst = reinterpret_cast<float4*>(out + (size_t)c * kWireChunk + kWireHdr + (size_t)s * kWireEnt);
  const float4 p = pos[i], q = rot[i], d = col_dims[i];
  const uint32_t shape = col_kind[i];
  float sx, sy, sz;
  uint32_t kind;
  if (shape == 0u) { sx = sy = sz = d.x; kind = 1u; }
  else if (shape == 1u) { sx = d.x; sy = d.y; sz = d.z; kind = 2u; }
  else { sx = d.x; sy = (d.y + d.x) * 0.5f; sz = d.x; kind = 3u; }
  dst[0] = make_float4(__uint_as_float(i + 1u), p.x, p.y, p.z);
  dst[1] = make_float4(q.x, q.y, q.z, q.w);
  dst[2] = make_float4(sx, sy, sz, __uint_as_float(kind));
}
// NetHdr (wire.rs:9-20), repr(C): magic u32, ver u16, kind u8, flags u8, tick u64, epoch u64,
// total u16, index u16, payload_len u32 -- 32 bytes.
__global__ void k_wire_hdrs(uint32_t nchunks, uint32_t nent, unsigned long long tick, unsigned long long epoch,
                            uint8_t* out) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nchunks) return;
  const uint32_t in_chunk = min(kWirePer, nent - c * kWirePer);
  uint4* dst = reinterpret_cast<uint4*>(out + (size_t)c * kWireChunk);
  dst[0] = make_uint4(kWireMagic, kWireVer | (kWireKindSnapshot << 16), (uint32_t)tick, (uint32_t)(tick >> 32));
  dst[1] = make_uint4((uint32_t)epoch, (uint32_t)(epoch >> 32), (nchunks & 0xFFFFu) | (c << 16), in_chunk * kWireEnt);
}

// Sizes of the snapshot of the live bodies; packs it into host_out when given (cap bytes).
void WorldGpu::pack_snapshot(unsigned long long tick, unsigned long long epoch, uint8_t* host_out, size_t cap,
                             size_t* bytes, uint32_t* chunks) {
  auto& S = *s_;
  cudaStream_t st = stream_;
  uint32_t nlive = 0;
  for (uint32_t i = 0; i < nb_; ++i) nlive += h_alive_[i] ? 1u : 0u;
  const uint32_t nch = (nlive + kWirePer - 1) / kWirePer;
  *chunks = nch;
  *bytes = (size_t)nch * kWireHdr + (size_t)nlive * kWireEnt;
  if (!host_out || nlive == 0) return;
  if (cap < *bytes) throw std::length_error("snapshot larger than the buffer");
  S.wire_flag.ensure(nb_ + 1);
  S.wire_off.ensure(nb_ + 1);
  S.wire_buf.ensure((size_t)nch * kWireChunk + 16);
  k_wire_flags<<<nblk(nb_), T, 0, st>>>(nb_, alive_d.p, S.wire_flag.p); RP_COUNT_LAUNCH(1);
  exclusive_scan_total(S, S.wire_flag.p, S.wire_off.p, nb_, st);
  k_wire_ents<<<nblk(nb_), T, 0, st>>>(nb_, alive_d.p, S.wire_off.p, pos.p, rot.p, col_kind.p, col_dims.p, S.wire_buf.p);
  RP_COUNT_LAUNCH(1);
  k_wire_hdrs<<<nblk(nch), T, 0, st>>>(nch, nlive, tick, epoch, S.wire_buf.p); RP_COUNT_LAUNCH(1);
  RP_CUDA(cudaMemcpyAsync(host_out, S.wire_buf.p, *bytes, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
}

}  // namespace rp
