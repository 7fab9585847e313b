// step_prims.cu -- device-wide sort / scan / select used between the step's kernels. All are
// stable and deterministic (LSD radix sort, integer scans), so the tick is bit-reproducible.
#include <cub/cub.cuh>

#include "step_internal.cuh"

namespace rp {

unsigned long long g_launches = 0;
thread_local cudaStream_t g_alloc_stream = nullptr;

namespace {
template <class F>
void with_tmp(WorldGpu::Scratch& S, F f) {
  size_t bytes = 0;
  f(nullptr, bytes);
  S.cub_tmp.ensure(bytes + 16);
  f(S.cub_tmp.p, bytes);
}
}  // namespace

void select_flagged_iota(WorldGpu::Scratch& S, int n, const uint32_t* flags, uint32_t* out, uint32_t* d_count,
                         cudaStream_t st) {
  cub::CountingInputIterator<uint32_t> it(0);
  with_tmp(S, [&](void* t, size_t& b) {
    RP_CUDA(cub::DeviceSelect::Flagged(t, b, it, flags, out, d_count, n, st));
  });
  RP_COUNT_LAUNCH(2);
}

uint32_t select_flagged_u64(WorldGpu::Scratch& S, const unsigned long long* in, const uint8_t* flags,
                            unsigned long long* out, uint32_t n, cudaStream_t st) {
  S.counts.ensure(4);
  with_tmp(S, [&](void* t, size_t& b) {
    RP_CUDA(cub::DeviceSelect::Flagged(t, b, in, flags, out, S.counts.p + 2, n, st));
  });
  RP_COUNT_LAUNCH(2);
  uint32_t c = 0;
  RP_CUDA(cudaMemcpyAsync(&c, S.counts.p + 2, 4, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
  return c;
}

uint32_t select_flagged_u32(WorldGpu::Scratch& S, const uint32_t* in, const uint8_t* flags, uint32_t* out,
                            uint32_t n, cudaStream_t st) {
  S.counts.ensure(4);
  with_tmp(S, [&](void* t, size_t& b) {
    RP_CUDA(cub::DeviceSelect::Flagged(t, b, in, flags, out, S.counts.p + 3, n, st));
  });
  RP_COUNT_LAUNCH(2);
  uint32_t c = 0;
  RP_CUDA(cudaMemcpyAsync(&c, S.counts.p + 3, 4, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
  return c;
}

void sort_pairs_u32(WorldGpu::Scratch& S, const uint32_t* kin, uint32_t* kout, const uint32_t* vin, uint32_t* vout,
                    uint32_t n, int bit0, int bit1, cudaStream_t st) {
  if (n == 0) return;
  with_tmp(S, [&](void* t, size_t& b) {
    RP_CUDA(cub::DeviceRadixSort::SortPairs(t, b, kin, kout, vin, vout, (int)n, bit0, bit1, st));
  });
  RP_COUNT_LAUNCH(1 + (bit1 - bit0 + 7) / 8);
}

void sort_pairs_u64(WorldGpu::Scratch& S, const unsigned long long* kin, unsigned long long* kout, const uint32_t* vin,
                    uint32_t* vout, uint32_t n, int bit0, int bit1, cudaStream_t st) {
  if (n == 0) return;
  with_tmp(S, [&](void* t, size_t& b) {
    RP_CUDA(cub::DeviceRadixSort::SortPairs(t, b, kin, kout, vin, vout, (int)n, bit0, bit1, st));
  });
  RP_COUNT_LAUNCH(1 + (bit1 - bit0 + 7) / 8);
}

void sort_keys_u64(WorldGpu::Scratch& S, const unsigned long long* kin, unsigned long long* kout, uint32_t n,
                   cudaStream_t st) {
  if (n == 0) return;
  with_tmp(S, [&](void* t, size_t& b) {
    RP_CUDA(cub::DeviceRadixSort::SortKeys(t, b, kin, kout, (int)n, 0, 64, st));
  });
  RP_COUNT_LAUNCH(9);
}

void exclusive_scan(WorldGpu::Scratch& S, const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t st) {
  if (n == 0) return;
  with_tmp(S, [&](void* t, size_t& b) {
    RP_CUDA(cub::DeviceScan::ExclusiveSum(t, b, in, out, (int)n, st));
  });
  RP_COUNT_LAUNCH(2);
}

// Exclusive sum of in[0, n) into out; returns the total (one device-to-host read).
uint32_t exclusive_scan_total(WorldGpu::Scratch& S, const uint32_t* in, uint32_t* out, uint32_t n, cudaStream_t st) {
  if (n == 0) return 0;
  exclusive_scan(S, in, out, n, st);
  uint32_t a = 0, b = 0;
  RP_CUDA(cudaMemcpyAsync(&a, out + n - 1, 4, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaMemcpyAsync(&b, in + n - 1, 4, cudaMemcpyDeviceToHost, st));
  RP_CUDA(cudaStreamSynchronize(st));
  return a + b;
}

}  // namespace rp
