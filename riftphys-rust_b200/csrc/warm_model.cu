// warm_model.cu -- the learned warm start: a small MLP (24 -> 128 -> 128 -> 128 -> 3, SiLU) that
// predicts each contact row's converged impulse (normal, two friction components) from local
// features, evaluated and trained on the 5th-generation tensor cores. Every matrix product runs
// through one kernel, k_tc_gemm: C[M x N] (f32) = A[M x K] . B[N x K]^T with A and B in bf16,
// both K-contiguous, issued as tcgen05.mma (kind::f16, f32 accumulate) by one elected thread with
// the accumulator in tensor memory and the operands staged in shared memory in the canonical
// no-swizzle K-major layout (8-row x 16-byte core matrices). The forward pass keeps each layer's
// pre-activation (f32) and activation (bf16); the backward pass is the same GEMM on transposed
// operands; Adam updates f32 master weights.
//
// Completion of the MMAs is signalled by tcgen05.commit on an mbarrier; every wait is bounded and
// sets an error flag (RPHYS_STATERR_WAIT_TIMEOUT) instead of spinning forever.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "warm_model.h"

namespace rp {

#define WM_CUDA(x)                                                                      \
  do {                                                                                  \
    cudaError_t e__ = (x);                                                              \
    if (e__ != cudaSuccess)                                                             \
      throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e__) + \
                               " at " __FILE__ ":" + std::to_string(__LINE__));         \
  } while (0)

extern unsigned long long g_launches;
static inline void wm_count(unsigned n) {
  g_launches += n;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA launch error: ") + cudaGetErrorString(e));
}

// ------------------------------------------------------------------ tcgen05 primitives
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle, K-major: start, leading (K-adjacent core matrices)
// and stride (8-row groups) byte offsets in 16-byte units, version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;  // version
  return d;                 // base offset 0, lbo mode 0, layout type 0 (no swizzle)
}
// Instruction descriptor for kind::f16: D f32, A and B bf16, both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t M, uint32_t N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}
__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}
// Bounded wait for the mbarrier phase with the given parity; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity) {
  uint32_t a = smem_u32(mbar);
  for (uint32_t i = 0; i < (1u << 26); ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// ------------------------------------------------------------------ the GEMM
// One CTA (128 threads) computes a 128 x NT tile of C; K is consumed in chunks of KC staged into
// shared memory (core-matrix layout: element (r, k) at (r/8)*SBO + (k/8)*128 + (r%8)*16 + (k%8)*2,
// SBO = KC/8 * 128), each chunk by KC/16 MMAs of 128 x NT x 16. Accumulator: NT f32 columns of TMEM.
#define TC_KC 64
template <int NT>
struct TcSmem {
  __nv_bfloat16 a[128 * TC_KC];
  __nv_bfloat16 b[NT * TC_KC];
  uint64_t mbar;
  uint32_t tmem;
};
template <int NT>
__global__ void __launch_bounds__(128) k_tc_gemm(uint32_t M, uint32_t N, uint32_t K, const __nv_bfloat16* __restrict__ A,
                                                 uint32_t lda, const __nv_bfloat16* __restrict__ Bm, uint32_t ldb,
                                                 float* C, uint32_t ldc, const float* __restrict__ bias, uint32_t* err) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  TcSmem<NT>& sm = *reinterpret_cast<TcSmem<NT>*>(tc_raw);
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t m0 = blockIdx.x * 128u, n0 = blockIdx.y * (uint32_t)NT;
  constexpr uint32_t NCOL = NT < 32 ? 32u : (uint32_t)NT;  // TMEM allocation: a power of two >= 32
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem)),
                 "r"(NCOL));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) mbar_init(&sm.mbar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem;
  const uint32_t idesc = umma_idesc(128u, (uint32_t)NT);
  const uint32_t SBO = (TC_KC / 8) * 128;
  bool ok = true;
  uint32_t phase = 0;
  for (uint32_t kc = 0; kc < K; kc += TC_KC) {
    const uint32_t kn = (K - kc) < (uint32_t)TC_KC ? (K - kc) : (uint32_t)TC_KC;  // multiple of 16
    // stage A (128 x kn) and B (NT x kn): one 16-byte piece (8 bf16 of one row) per step
    const uint32_t pieces_a = 128u * (kn / 8u), pieces_b = (uint32_t)NT * (kn / 8u);
    for (uint32_t p = tid; p < pieces_a; p += 128) {
      uint32_t r = p / (kn / 8u), j = p % (kn / 8u);
      uint4 v = make_uint4(0, 0, 0, 0);
      if (m0 + r < M) v = *reinterpret_cast<const uint4*>(A + (size_t)(m0 + r) * lda + kc + 8u * j);
      *reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(sm.a) + (r / 8u) * SBO + j * 128u + (r % 8u) * 16u) = v;
    }
    for (uint32_t p = tid; p < pieces_b; p += 128) {
      uint32_t r = p / (kn / 8u), j = p % (kn / 8u);
      uint4 v = make_uint4(0, 0, 0, 0);
      if (n0 + r < N) v = *reinterpret_cast<const uint4*>(Bm + (size_t)(n0 + r) * ldb + kc + 8u * j);
      *reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(sm.b) + (r / 8u) * SBO + j * 128u + (r % 8u) * 16u) = v;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      const uint32_t a0 = smem_u32(sm.a), b0 = smem_u32(sm.b);
      for (uint32_t ks = 0; ks < kn / 16u; ++ks)
        umma_bf16(tmem, umma_desc(a0 + ks * 256u, 128u, SBO), umma_desc(b0 + ks * 256u, 128u, SBO), idesc,
                  (kc > 0 || ks > 0) ? 1u : 0u);
      umma_commit(&sm.mbar);
    }
    const bool waited = mbar_wait(&sm.mbar, phase);
    phase ^= 1u;
    tc_fence_after();
    if (!__syncthreads_and(waited)) { ok = false; break; }  // the same decision in every thread
  }
  if (!ok) {
    if (tid == 0) {
      atomicOr(err, 4u);  // RPHYS_STATERR_WAIT_TIMEOUT
      mbar_wait(&sm.mbar, phase ^ 1u);  // give an MMA still in flight one more bounded chance
    }
  } else {
    // epilogue: thread t owns row m0 + t (TMEM lane t), 16 columns per load
    const uint32_t row = m0 + warp * 32u + lane;
    for (uint32_t c = 0; c < (uint32_t)NT; c += 16) {
      float v[16];
      tmem_ld16(tmem + ((warp * 32u) << 16) + c, v);
      if (row < M)
        for (int k = 0; k < 16; ++k) {
          uint32_t col = n0 + c + (uint32_t)k;
          if (col < N) C[(size_t)row * ldc + col] = v[k] + (bias ? bias[col] : 0.0f);
        }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOL));
}

// C = A . B^T (+ bias per column). M % 128 == 0, N % 16 == 0, K % 16 == 0, lda/ldb % 8 == 0.
void tc_gemm(uint32_t M, uint32_t N, uint32_t K, const __nv_bfloat16* A, uint32_t lda, const __nv_bfloat16* B, uint32_t ldb,
             float* C, uint32_t ldc, const float* bias, uint32_t* err, cudaStream_t st) {
  if (M % 128 || N % 16 || K % 16 || lda % 8 || ldb % 8) throw std::invalid_argument("tc_gemm: unsupported shape");
  if (N >= 128 && N % 128 == 0) {
    dim3 grid(M / 128, N / 128);
    size_t sm = sizeof(TcSmem<128>) + 1024;
    static bool attr = false;
    if (!attr) { WM_CUDA(cudaFuncSetAttribute(k_tc_gemm<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(64 << 10))); attr = true; }
    // 64 KB per CTA keeps at most three on an SM: their TMEM (128 columns each) always fits
    k_tc_gemm<128><<<grid, 128, 64 << 10, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, err);
    (void)sm;
  } else {
    dim3 grid(M / 128, (N + 15) / 16);
    static bool attr = false;
    if (!attr) { WM_CUDA(cudaFuncSetAttribute(k_tc_gemm<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(64 << 10))); attr = true; }
    k_tc_gemm<16><<<grid, 128, 64 << 10, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, err);
  }
  wm_count(1);
}

// ------------------------------------------------------------------ fused inference
// The whole forward pass in one kernel: a persistent CTA of 128 threads keeps the four bf16 weight
// matrices in shared memory (core-matrix layout, staged once), and for each tile of 128 rows converts
// the rows' 24 f32 features to bf16, then per layer issues the MMAs into one 128-column TMEM
// accumulator and runs the epilogue -- thread t reads row t's columns (tcgen05.ld), adds the bias,
// applies SiLU and writes the bf16 activation into shared memory as the next layer's A operand.
// The last layer writes the three outputs. Every product and rounding is the one the layer-by-layer
// path (forward) makes, so the outputs are the same bits. Waits are bounded: a timeout sets
// RPHYS_STATERR_WAIT_TIMEOUT in *err and the CTA stops.
namespace fused {
constexpr uint32_t kIn = 24, kInPad = 32, kH = 128;
// byte offset of element (r, k) of a [rows x K] operand in the no-swizzle K-major layout
__device__ __forceinline__ uint32_t core_off(uint32_t r, uint32_t k, uint32_t K) {
  return (r / 8u) * (K / 8u) * 128u + (k / 8u) * 128u + (r % 8u) * 16u + (k % 8u) * 2u;
}
struct Smem {
  __nv_bfloat16 w1[kH * kInPad], w2[kH * kH], w3[kH * kH], w4[16 * kH];
  __nv_bfloat16 x[128 * kInPad], a[128 * kH];
  float b[3 * kH + 16];
  uint64_t mbar;
  uint32_t tmem;
};
}  // namespace fused
__global__ void __launch_bounds__(128) k_mlp_fused(uint32_t n, const float* __restrict__ feats,
                                                   const __nv_bfloat16* __restrict__ wb, const float* __restrict__ w32,
                                                   float* out3, uint32_t* err, uint32_t oW1, uint32_t oW2, uint32_t oW3,
                                                   uint32_t oW4, uint32_t oB1, uint32_t oB2, uint32_t oB3, uint32_t oB4) {
  using namespace fused;
  extern __shared__ __align__(1024) unsigned char mf_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(mf_raw);
  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sm.tmem)), "r"(kH));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) mbar_init(&sm.mbar, 1);
  // weights into the core-matrix layout, one 16-byte piece (8 bf16 of one row) per step
  auto stage = [&](__nv_bfloat16* dst, const __nv_bfloat16* src, uint32_t rows, uint32_t K) {
    for (uint32_t p = tid; p < rows * (K / 8u); p += 128u) {
      uint32_t r = p / (K / 8u), j = p % (K / 8u);
      *reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(dst) + core_off(r, 8u * j, K)) =
          *reinterpret_cast<const uint4*>(src + (size_t)r * K + 8u * j);
    }
  };
  stage(sm.w1, wb + oW1, kH, kInPad);
  stage(sm.w2, wb + oW2, kH, kH);
  stage(sm.w3, wb + oW3, kH, kH);
  stage(sm.w4, wb + oW4, 16, kH);
  for (uint32_t i = tid; i < kH; i += 128u) {
    sm.b[i] = w32[oB1 + i]; sm.b[kH + i] = w32[oB2 + i]; sm.b[2 * kH + i] = w32[oB3 + i];
  }
  if (tid < 16) sm.b[3 * kH + tid] = w32[oB4 + tid];
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = sm.tmem;
  uint32_t phase = 0;
  bool ok = true;
  // one layer: D[128 x N] = A[128 x K] . W^T, then wait for it
  auto layer = [&](const __nv_bfloat16* A, const __nv_bfloat16* W, uint32_t N, uint32_t K) {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      const uint32_t a0 = smem_u32(A), b0 = smem_u32(W), sbo = (K / 8u) * 128u, idesc = umma_idesc(128u, N);
      for (uint32_t ks = 0; ks < K / 16u; ++ks)
        umma_bf16(tmem, umma_desc(a0 + ks * 256u, 128u, sbo), umma_desc(b0 + ks * 256u, 128u, sbo), idesc, ks ? 1u : 0u);
      umma_commit(&sm.mbar);
    }
    const bool waited = mbar_wait(&sm.mbar, phase);
    phase ^= 1u;
    tc_fence_after();
    return __syncthreads_and(waited) != 0;
  };
  const uint32_t tiles = (n + 127u) / 128u;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const uint32_t row = tile * 128u + tid;  // thread t: row t of the tile (TMEM lane t)
    // features: f32 -> bf16, inputs 24..31 zero, rows past n zero
    for (uint32_t j = 0; j < kInPad / 8u; ++j) {
      __align__(16) __nv_bfloat16 v[8];
      for (uint32_t q = 0; q < 8u; ++q) {
        uint32_t k = 8u * j + q;
        v[q] = __float2bfloat16(row < n && k < kIn ? feats[(size_t)row * kIn + k] : 0.0f);
      }
      *reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(sm.x) + core_off(tid, 8u * j, kInPad)) =
          *reinterpret_cast<const uint4*>(v);
    }
    const __nv_bfloat16* Ws[3] = {sm.w1, sm.w2, sm.w3};
    for (int L = 0; L < 3 && ok; ++L) {
      ok = layer(L == 0 ? sm.x : sm.a, Ws[L], kH, L == 0 ? kInPad : kH);
      if (!ok) break;
      // epilogue: bias + SiLU -> bf16 activation (the next layer's A operand, row t)
      for (uint32_t c = 0; c < kH; c += 16u) {
        float v[16];
        tmem_ld16(tmem + ((warp * 32u) << 16) + c, v);
        __align__(16) __nv_bfloat16 h[16];
        for (int k = 0; k < 16; ++k) {
          float z = v[k] + sm.b[L * kH + c + k];
          h[k] = __float2bfloat16(z / (1.0f + expf(-z)));
        }
        unsigned char* base = reinterpret_cast<unsigned char*>(sm.a);
        *reinterpret_cast<uint4*>(base + core_off(tid, c, kH)) = *reinterpret_cast<const uint4*>(h);
        *reinterpret_cast<uint4*>(base + core_off(tid, c + 8u, kH)) = *reinterpret_cast<const uint4*>(h + 8);
      }
      tc_fence_before();  // the TMEM reads are done before the next layer's MMAs overwrite the columns
    }
    if (!ok) break;
    ok = layer(sm.a, sm.w4, 16u, kH);
    if (!ok) break;
    float v[16];
    tmem_ld16(tmem + ((warp * 32u) << 16), v);
    if (row < n)
      for (int k = 0; k < 3; ++k) out3[(size_t)row * 3 + k] = v[k] + sm.b[3 * kH + k];
    tc_fence_before();
    __syncthreads();  // the accumulator is read before the next tile's MMAs
    tc_fence_after();
  }
  if (!ok && tid == 0) {
    atomicOr(err, 4u);  // RPHYS_STATERR_WAIT_TIMEOUT
    mbar_wait(&sm.mbar, phase ^ 1u);  // an MMA still in flight gets one more bounded chance
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kH));
}

// ------------------------------------------------------------------ elementwise pieces
__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}
// H = bf16(SiLU(Z)) over an M x N f32 matrix (row stride ldz) into ldh
__global__ void k_silu_bf16(uint32_t M, uint32_t N, const float* __restrict__ Z, uint32_t ldz, __nv_bfloat16* H, uint32_t ldh) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)M * N) return;
  uint32_t r = (uint32_t)(i / N), c = (uint32_t)(i % N);
  H[(size_t)r * ldh + c] = __float2bfloat16(silu(Z[(size_t)r * ldz + c]));
}
// G = bf16(dH * SiLU'(Z))
__global__ void k_dsilu_bf16(uint32_t M, uint32_t N, const float* __restrict__ dH, const float* __restrict__ Z,
                             __nv_bfloat16* G) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)M * N) return;
  G[i] = __float2bfloat16(dH[i] * dsilu(Z[i]));
}
// bf16 transpose of an R x C matrix (row stride ld) into C x R
__global__ void k_transpose_bf16(uint32_t R, uint32_t C, const __nv_bfloat16* __restrict__ X, uint32_t ld, __nv_bfloat16* Y,
                                 uint32_t ldy) {
  __shared__ __nv_bfloat16 t[32][33];
  uint32_t bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (uint32_t k = threadIdx.y; k < 32; k += blockDim.y) {
    uint32_t r = by + k, c = bx + threadIdx.x;
    t[k][threadIdx.x] = (r < R && c < C) ? X[(size_t)r * ld + c] : __float2bfloat16(0.0f);
  }
  __syncthreads();
  for (uint32_t k = threadIdx.y; k < 32; k += blockDim.y) {
    uint32_t c = bx + k, r = by + threadIdx.x;
    if (c < C && r < R) Y[(size_t)c * ldy + r] = t[threadIdx.x][k];
  }
}
__global__ void k_f32_to_bf16(size_t n, const float* __restrict__ x, __nv_bfloat16* y) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16(x[i]);
}
// column sums of an M x N f32 matrix (bias gradients), one thread per column, fixed order
__global__ void k_colsum(uint32_t M, uint32_t N, const float* __restrict__ X, uint32_t ldx, float* out) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  float s = 0.0f;
  for (uint32_t r = 0; r < M; ++r) s += X[(size_t)r * ldx + c];
  out[c] = s;
}
// output gradient of the mean squared error over the 3 used outputs (the 16-wide padding stays 0)
__global__ void k_mse_grad(uint32_t M, uint32_t n_valid, const float* __restrict__ Y, const float* __restrict__ T, float scale,
                           float* dY, float* loss) {
  uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= M) return;
  float l = 0.0f;
  for (int c = 0; c < 16; ++c) {
    float g = 0.0f;
    if (c < 3 && r < n_valid) {
      float d = Y[(size_t)r * 16 + c] - T[(size_t)r * 3 + c];
      g = 2.0f * d * scale;
      l += d * d;
    }
    dY[(size_t)r * 16 + c] = g;
  }
  if (r < n_valid && loss) atomicAdd(loss, l * scale);
}
__global__ void k_adam(uint32_t n, float* w, const float* __restrict__ g, float* m, float* v, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i];
  m[i] = b1 * m[i] + (1.0f - b1) * gi;
  v[i] = b2 * v[i] + (1.0f - b2) * gi * gi;
  w[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

static inline unsigned blocks(size_t n, unsigned t = 256) { return (unsigned)((n + t - 1) / t); }

// ------------------------------------------------------------------ the model
WarmModel::WarmModel(uint64_t seed) {
  WM_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
  WM_CUDA(cudaMalloc(&err_, 4));
  WM_CUDA(cudaMemset(err_, 0, 4));
  // He-uniform initialisation from a splitmix64 stream (deterministic per seed)
  std::vector<float> w(kParams, 0.0f);
  uint64_t s = seed;
  auto next = [&]() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](uint32_t off, uint32_t rows, uint32_t cols, uint32_t fan_in) {
    double a = std::sqrt(6.0 / fan_in);
    for (uint32_t r = 0; r < rows; ++r)
      for (uint32_t c = 0; c < cols; ++c) w[off + r * cols + c] = (float)((2.0 * next() - 1.0) * a);
  };
  fill(kW1, kH, kInPad, kIn);
  fill(kW2, kH, kH, kH);
  fill(kW3, kH, kH, kH);
  fill(kW4, 3, kH, kH);  // rows 3..15 of W4 stay 0 (padding)
  for (uint32_t r = 0; r < kH; ++r)
    for (uint32_t c = kIn; c < kInPad; ++c) w[kW1 + r * kInPad + c] = 0.0f;
  WM_CUDA(cudaMalloc(&w_, 4 * kParams));
  WM_CUDA(cudaMalloc(&g_, 4 * kParams));
  WM_CUDA(cudaMalloc(&m_, 4 * kParams));
  WM_CUDA(cudaMalloc(&v_, 4 * kParams));
  WM_CUDA(cudaMalloc(&wb_, 2 * kParams));
  WM_CUDA(cudaMalloc(&wt_, 2 * (size_t)kH * kH * 3));
  WM_CUDA(cudaMemcpy(w_, w.data(), 4 * kParams, cudaMemcpyHostToDevice));
  WM_CUDA(cudaMemset(m_, 0, 4 * kParams));
  WM_CUDA(cudaMemset(v_, 0, 4 * kParams));
  refresh_bf16();
}
WarmModel::~WarmModel() {
  cudaStreamSynchronize(st_);
  for (void* p : {(void*)w_, (void*)g_, (void*)m_, (void*)v_, (void*)wb_, (void*)wt_, (void*)err_}) cudaFree(p);
  for (auto& b : bufs_) cudaFree(b.p);
  cudaStreamDestroy(st_);
}
void* WarmModel::buf(int k, size_t bytes) {
  if (bufs_.size() <= (size_t)k) bufs_.resize(k + 1);
  Buf& b = bufs_[k];
  if (b.bytes < bytes) {
    if (b.p) WM_CUDA(cudaFree(b.p));
    WM_CUDA(cudaMalloc(&b.p, bytes));
    b.bytes = bytes;
  }
  return b.p;
}
// bf16 copies of the weights, and the transposes the backward pass multiplies by
void WarmModel::refresh_bf16() {
  k_f32_to_bf16<<<blocks(kParams), 256, 0, st_>>>(kParams, w_, wb_); wm_count(1);
  dim3 tb(32, 8);
  // W2^T, W3^T (128 x 128) and W4^T (128 x 16): rows of the transposed matrix are the inputs
  k_transpose_bf16<<<dim3(kH / 32, kH / 32), tb, 0, st_>>>(kH, kH, wb_ + kW2, kH, wt_, kH); wm_count(1);
  k_transpose_bf16<<<dim3(kH / 32, kH / 32), tb, 0, st_>>>(kH, kH, wb_ + kW3, kH, wt_ + kH * kH, kH); wm_count(1);
  k_transpose_bf16<<<dim3(kH / 32, 1), tb, 0, st_>>>(16, kH, wb_ + kW4, kH, wt_ + 2 * kH * kH, 16); wm_count(1);
}
void WarmModel::check_err() {
  uint32_t e = 0;
  WM_CUDA(cudaMemcpyAsync(&e, err_, 4, cudaMemcpyDeviceToHost, st_));
  WM_CUDA(cudaStreamSynchronize(st_));
  if (e) throw std::runtime_error("warm model: a tensor-core wait timed out");
}

// Forward over M rows (M % 128 == 0) of bf16 features X [M x 32]: Z1..Z3 (f32), H1..H3 (bf16), Y [M x 16].
void WarmModel::forward(uint32_t M, const __nv_bfloat16* X, float* Y, cudaStream_t st, Acts* a) {
  float* Z1 = a->Z[0]; float* Z2 = a->Z[1]; float* Z3 = a->Z[2];
  __nv_bfloat16 *H1 = a->H[0], *H2 = a->H[1], *H3 = a->H[2];
  const size_t n = (size_t)M * kH;
  tc_gemm(M, kH, kInPad, X, kInPad, wb_ + kW1, kInPad, Z1, kH, w_ + kB1, err_, st);
  k_silu_bf16<<<blocks(n), 256, 0, st>>>(M, kH, Z1, kH, H1, kH); wm_count(1);
  tc_gemm(M, kH, kH, H1, kH, wb_ + kW2, kH, Z2, kH, w_ + kB2, err_, st);
  k_silu_bf16<<<blocks(n), 256, 0, st>>>(M, kH, Z2, kH, H2, kH); wm_count(1);
  tc_gemm(M, kH, kH, H2, kH, wb_ + kW3, kH, Z3, kH, w_ + kB3, err_, st);
  k_silu_bf16<<<blocks(n), 256, 0, st>>>(M, kH, Z3, kH, H3, kH); wm_count(1);
  tc_gemm(M, 16, kH, H3, kH, wb_ + kW4, kH, Y, 16, w_ + kB4, err_, st);
}
WarmModel::Acts WarmModel::acts(uint32_t M, int base) {
  Acts a;
  for (int k = 0; k < 3; ++k) {
    a.Z[k] = (float*)buf(base + k, 4 * (size_t)M * kH);
    a.H[k] = (__nv_bfloat16*)buf(base + 3 + k, 2 * (size_t)M * kH);
  }
  return a;
}

// The fused forward pass (k_mlp_fused) over n rows of device features into device out3, queued on
// st with nothing waited for; a timed-out wait ORs RPHYS_STATERR_WAIT_TIMEOUT into *err.
void WarmModel::predict_async(uint32_t n, const float* feats, float* out3, uint32_t* err, cudaStream_t st) {
  if (!n) return;
  static int attr_dev = -1;
  int dev = 0;
  WM_CUDA(cudaGetDevice(&dev));
  if (attr_dev != dev) {
    WM_CUDA(cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(fused::Smem)));
    attr_dev = dev;
  }
  int sms = 148;
  WM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const uint32_t tiles = (n + 127) / 128;
  const uint32_t grid = tiles < (uint32_t)sms ? tiles : (uint32_t)sms;  // one persistent CTA per SM
  k_mlp_fused<<<grid, 128, sizeof(fused::Smem), st>>>(n, feats, wb_, w_, out3, err, kW1, kW2, kW3, kW4, kB1, kB2, kB3, kB4);
  wm_count(1);
}
// Predictions for n rows of f32 features (24 each, host or device pointer given by on_device),
// returned when they are done.
void WarmModel::predict(uint32_t n, const float* feats, float* out3, bool on_device, cudaStream_t st) {
  if (!st) st = st_;
  if (n == 0) return;
  const float* F = feats;
  float* O = out3;
  if (!on_device) {
    float* f = (float*)buf(0, 4 * (size_t)n * kIn);
    WM_CUDA(cudaMemcpyAsync(f, feats, 4 * (size_t)n * kIn, cudaMemcpyHostToDevice, st));
    F = f;
    O = (float*)buf(2, 12 * (size_t)n);
  }
  predict_async(n, F, O, err_, st);
  if (!on_device) WM_CUDA(cudaMemcpyAsync(out3, O, 12 * (size_t)n, cudaMemcpyDeviceToHost, st));
  WM_CUDA(cudaStreamSynchronize(st));
  check_err();
}

// One forward/backward pass over n rows (host arrays): gradients into g_ (f32, the weight layout),
// loss returned. The batch is padded to a multiple of 128 with zero rows that carry no loss.
float WarmModel::gradients(uint32_t n, const float* feats, const float* targets, bool on_device) {
  cudaStream_t st = st_;
  uint32_t M = (n + 127) / 128 * 128;
  float* F = (float*)buf(0, 4 * (size_t)M * kInPad);
  __nv_bfloat16* X = (__nv_bfloat16*)buf(1, 2 * (size_t)M * kInPad);
  float* Y = (float*)buf(2, 4 * (size_t)M * 16);
  float* T = (float*)buf(3, 4 * (size_t)M * 3);
  float* dY = (float*)buf(4, 4 * (size_t)M * 16);
  float* loss = (float*)buf(5, 16);
  WM_CUDA(cudaMemsetAsync(F, 0, 4 * (size_t)M * kInPad, st));
  WM_CUDA(cudaMemcpy2DAsync(F, 4 * kInPad, feats, 4 * kIn, 4 * kIn, n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  WM_CUDA(cudaMemsetAsync(T, 0, 4 * (size_t)M * 3, st));
  WM_CUDA(cudaMemcpyAsync(T, targets, 12 * (size_t)n, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
  WM_CUDA(cudaMemsetAsync(loss, 0, 4, st));
  k_f32_to_bf16<<<blocks((size_t)M * kInPad), 256, 0, st>>>((size_t)M * kInPad, F, X); wm_count(1);
  Acts a = acts(M, 8);
  forward(M, X, Y, st, &a);
  const float scale = 1.0f / (3.0f * (float)n);
  k_mse_grad<<<blocks(M), 256, 0, st>>>(M, n, Y, T, scale, dY, loss); wm_count(1);
  // buffers for the backward pass
  __nv_bfloat16* dYb = (__nv_bfloat16*)buf(20, 2 * (size_t)M * 16);
  __nv_bfloat16* dYt = (__nv_bfloat16*)buf(21, 2 * (size_t)M * 16);
  __nv_bfloat16* Ht = (__nv_bfloat16*)buf(22, 2 * (size_t)M * kH);
  __nv_bfloat16* Gb = (__nv_bfloat16*)buf(23, 2 * (size_t)M * kH);
  __nv_bfloat16* Gt = (__nv_bfloat16*)buf(24, 2 * (size_t)M * kH);
  float* dH = (float*)buf(25, 4 * (size_t)M * kH);
  float* dWt = (float*)buf(26, 4 * (size_t)kH * kH);
  __nv_bfloat16* Xt = (__nv_bfloat16*)buf(27, 2 * (size_t)M * kInPad);
  dim3 tb(32, 8);
  auto transpose = [&](uint32_t R, uint32_t Cc, const __nv_bfloat16* src, uint32_t ld, __nv_bfloat16* dst) {
    k_transpose_bf16<<<dim3((Cc + 31) / 32, (R + 31) / 32), tb, 0, st>>>(R, Cc, src, ld, dst, R); wm_count(1);
  };
  // output layer: dW4^T [128 x 16] = H3^T . dY, db4 = colsum(dY), dH3 = dY . W4
  k_f32_to_bf16<<<blocks((size_t)M * 16), 256, 0, st>>>((size_t)M * 16, dY, dYb); wm_count(1);
  transpose(M, 16, dYb, 16, dYt);
  transpose(M, kH, a.H[2], kH, Ht);
  tc_gemm(kH, 16, M, Ht, M, dYt, M, dWt, 16, nullptr, err_, st);
  k_transpose_f32(kH, 16, dWt, 16, g_ + kW4, kH, st);
  k_colsum<<<1, 32, 0, st>>>(M, 16, dY, 16, g_ + kB4); wm_count(1);
  tc_gemm(M, kH, 16, dYb, 16, wt_ + 2 * kH * kH, 16, dH, kH, nullptr, err_, st);
  // hidden layers 3, 2: G = dH * SiLU'(Z); dW = G^T . H_prev; db = colsum(G); dH_prev = G . W
  for (int layer = 2; layer >= 1; --layer) {
    k_dsilu_bf16<<<blocks((size_t)M * kH), 256, 0, st>>>(M, kH, dH, a.Z[layer], Gb); wm_count(1);
    float* Gf = (float*)buf(28, 4 * (size_t)M * kH);
    k_bf16_to_f32((size_t)M * kH, Gb, Gf, st);
    k_colsum<<<1, 128, 0, st>>>(M, kH, Gf, kH, g_ + (layer == 2 ? kB3 : kB2)); wm_count(1);
    transpose(M, kH, Gb, kH, Gt);
    transpose(M, kH, a.H[layer - 1], kH, Ht);
    tc_gemm(kH, kH, M, Gt, M, Ht, M, g_ + (layer == 2 ? kW3 : kW2), kH, nullptr, err_, st);
    tc_gemm(M, kH, kH, Gb, kH, wt_ + (layer == 2 ? kH * kH : 0), kH, dH, kH, nullptr, err_, st);
  }
  // first layer: G1 = dH1 * SiLU'(Z1); dW1 = G1^T . X; db1 = colsum(G1)
  k_dsilu_bf16<<<blocks((size_t)M * kH), 256, 0, st>>>(M, kH, dH, a.Z[0], Gb); wm_count(1);
  float* Gf = (float*)buf(28, 4 * (size_t)M * kH);
  k_bf16_to_f32((size_t)M * kH, Gb, Gf, st);
  k_colsum<<<1, 128, 0, st>>>(M, kH, Gf, kH, g_ + kB1); wm_count(1);
  transpose(M, kH, Gb, kH, Gt);
  transpose(M, kInPad, X, kInPad, Xt);
  tc_gemm(kH, kInPad, M, Gt, M, Xt, M, g_ + kW1, kInPad, nullptr, err_, st);
  float l = 0.0f;
  WM_CUDA(cudaMemcpyAsync(&l, loss, 4, cudaMemcpyDeviceToHost, st));
  WM_CUDA(cudaStreamSynchronize(st));
  check_err();
  return l;
}

void WarmModel::adam_step(float lr) {
  step_++;
  const float b1 = 0.9f, b2 = 0.999f;
  float c1 = 1.0f - std::pow(b1, (float)step_), c2 = 1.0f - std::pow(b2, (float)step_);
  k_adam<<<blocks(kParams), 256, 0, st_>>>(kParams, w_, g_, m_, v_, lr, b1, b2, 1e-8f, c1, c2); wm_count(1);
  // the padding of W1 (inputs 24..31) and of W4 (outputs 3..15) stays zero
  refresh_bf16();
}

// Mini-batch Adam over n rows for `epochs` passes in a fixed order (batch b = rows [b*bs, ...)).
float WarmModel::train(uint32_t n, const float* feats, const float* targets, uint32_t epochs, uint32_t bs, float lr) {
  float* F = (float*)buf(40, 4 * (size_t)n * kIn + 16);
  float* T = (float*)buf(41, 12 * (size_t)n + 16);
  WM_CUDA(cudaMemcpyAsync(F, feats, 4 * (size_t)n * kIn, cudaMemcpyHostToDevice, st_));
  WM_CUDA(cudaMemcpyAsync(T, targets, 12 * (size_t)n, cudaMemcpyHostToDevice, st_));
  float last = 0.0f;
  for (uint32_t e = 0; e < epochs; ++e) {
    double sum = 0.0;
    uint32_t nb = 0;
    for (uint32_t b0 = 0; b0 < n; b0 += bs) {
      uint32_t m = n - b0 < bs ? n - b0 : bs;
      sum += gradients(m, F + (size_t)b0 * kIn, T + (size_t)b0 * 3, true);
      nb++;
      adam_step(lr);
    }
    last = (float)(sum / (nb ? nb : 1));
  }
  return last;
}

void WarmModel::get_weights(float* out) {
  WM_CUDA(cudaMemcpyAsync(out, w_, 4 * kParams, cudaMemcpyDeviceToHost, st_));
  WM_CUDA(cudaStreamSynchronize(st_));
}
void WarmModel::set_weights(const float* in) {
  WM_CUDA(cudaMemcpyAsync(w_, in, 4 * kParams, cudaMemcpyHostToDevice, st_));
  refresh_bf16();
  WM_CUDA(cudaStreamSynchronize(st_));
}
void WarmModel::get_grads(float* out) {
  WM_CUDA(cudaMemcpyAsync(out, g_, 4 * kParams, cudaMemcpyDeviceToHost, st_));
  WM_CUDA(cudaStreamSynchronize(st_));
}

__global__ void k_transpose_f32_kernel(uint32_t R, uint32_t C, const float* __restrict__ X, uint32_t ld, float* Y, uint32_t ldy) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R * C) return;
  uint32_t r = i / C, c = i % C;
  Y[(size_t)c * ldy + r] = X[(size_t)r * ld + c];
}
void k_transpose_f32(uint32_t R, uint32_t C, const float* X, uint32_t ld, float* Y, uint32_t ldy, cudaStream_t st) {
  k_transpose_f32_kernel<<<blocks((size_t)R * C), 256, 0, st>>>(R, C, X, ld, Y, ldy); wm_count(1);
}
__global__ void k_bf16_to_f32_kernel(size_t n, const __nv_bfloat16* __restrict__ x, float* y) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __bfloat162float(x[i]);
}
void k_bf16_to_f32(size_t n, const __nv_bfloat16* x, float* y, cudaStream_t st) {
  k_bf16_to_f32_kernel<<<blocks(n), 256, 0, st>>>(n, x, y); wm_count(1);
}

}  // namespace rp
