// warm_model.h -- the learned warm-start model (warm_model.cu): weights, training and inference.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace rp {

void tc_gemm(uint32_t M, uint32_t N, uint32_t K, const __nv_bfloat16* A, uint32_t lda, const __nv_bfloat16* B, uint32_t ldb,
             float* C, uint32_t ldc, const float* bias, uint32_t* err, cudaStream_t st);
void k_transpose_f32(uint32_t R, uint32_t C, const float* X, uint32_t ld, float* Y, uint32_t ldy, cudaStream_t st);
void k_bf16_to_f32(size_t n, const __nv_bfloat16* x, float* y, cudaStream_t st);

class WarmModel {
 public:
  // 24 features (padded to 32 columns), three hidden layers of 128, 3 outputs (padded to 16).
  // f32 master weights, one array: W1 [128 x 32] b1 [128] W2 [128 x 128] b2 W3 [128 x 128] b3
  // W4 [16 x 128] b4 [16] (rows 3..15 of W4 and inputs 24..31 of W1 are padding, kept at 0).
  static constexpr uint32_t kIn = 24, kInPad = 32, kH = 128;
  static constexpr uint32_t kW1 = 0, kB1 = kW1 + kH * kInPad, kW2 = kB1 + kH, kB2 = kW2 + kH * kH, kW3 = kB2 + kH,
                            kB3 = kW3 + kH * kH, kW4 = kB3 + kH, kB4 = kW4 + 16 * kH, kParams = kB4 + 16;
  static_assert(kW2 % 8 == 0 && kW3 % 8 == 0 && kW4 % 8 == 0, "bf16 weight blocks start on 16-byte boundaries");

  explicit WarmModel(uint64_t seed);
  ~WarmModel();
  void predict(uint32_t n, const float* feats, float* out3, bool on_device, cudaStream_t st = nullptr);
  // the same predictions from device features into device memory, queued on st without waiting
  void predict_async(uint32_t n, const float* feats, float* out3, uint32_t* err, cudaStream_t st);
  float gradients(uint32_t n, const float* feats, const float* targets, bool on_device);
  float train(uint32_t n, const float* feats, const float* targets, uint32_t epochs, uint32_t batch, float lr);
  void get_weights(float* out);
  void set_weights(const float* in);
  void get_grads(float* out);

 private:
  struct Acts { float* Z[3]; __nv_bfloat16* H[3]; };
  struct Buf { void* p = nullptr; size_t bytes = 0; };
  void forward(uint32_t M, const __nv_bfloat16* X, float* Y, cudaStream_t st, Acts* a);
  Acts acts(uint32_t M, int base);
  void* buf(int k, size_t bytes);
  void refresh_bf16();
  void adam_step(float lr);
  void check_err();
  cudaStream_t st_ = nullptr;
  float *w_ = nullptr, *g_ = nullptr, *m_ = nullptr, *v_ = nullptr;
  __nv_bfloat16 *wb_ = nullptr, *wt_ = nullptr;
  uint32_t* err_ = nullptr;
  uint64_t step_ = 0;
  std::vector<Buf> bufs_;
};

}  // namespace rp
