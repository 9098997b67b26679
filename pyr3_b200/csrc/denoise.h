// Denoiser kernels (C5 learned denoiser): the layers of a U-Net over NCHW
// f32 tensors and their adjoints.  Every tensor operand is (pointer,
// per-image stride): a channel slice of a larger tensor -- the U-Net's skip
// concatenation -- is a valid operand, so no layer copies.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pyr3 {

// out[n, co] = bias[co] + sum_ci conv3x3(in[n, ci], w[co, ci]), zero
// padding, optional ReLU.  w is [co][ci][3][3]; bias may be null.
cudaError_t dn_conv3x3(const float* in, int64_t in_ns, int ci, float* out, int64_t out_ns, int co,
                       int n, int h, int w, const float* weight, const float* bias, bool relu,
                       cudaStream_t s);
// The same convolution on the tensor cores (tcgen05): inputs and weights
// rounded to bf16, f32 accumulation; co <= 128.
cudaError_t dn_conv3x3_bf16(const float* in, int64_t in_ns, int ci, float* out, int64_t out_ns, int co,
                            int n, int h, int w, const float* weight, const float* bias, bool relu,
                            cudaStream_t s);
// dw[co, ci, k] = sum over images and pixels of dout[co] * shifted in[ci];
// db[co] = sum of dout[co] (db may be null).  Overwrites dw / db.  The sum
// is split over 32 pixel chunks whose partials go to scratch
// (dn_wgrad_scratch_floats(co, ci) floats) and are added in a fixed order.
size_t dn_wgrad_scratch_floats(int co, int ci);
cudaError_t dn_conv3x3_wgrad(const float* in, int64_t in_ns, int ci, const float* dout,
                             int64_t dout_ns, int co, int n, int h, int w, float* dw, float* db,
                             float* scratch, cudaStream_t s);
// The same gradients on the tensor cores (tcgen05): per tap a GEMM over the
// padded grid's positions with bf16 operands and f32 accumulation; co <= 128,
// ci <= 128, n <= 32; the same scratch.
cudaError_t dn_conv3x3_wgrad_bf16(const float* in, int64_t in_ns, int ci, const float* dout,
                                  int64_t dout_ns, int co, int n, int h, int w, float* dw, float* db,
                                  float* scratch, cudaStream_t s);
// wt[ci][co][k] = w[co][ci][8 - k]: the data gradient of a 3x3 convolution
// is the convolution of dout with these weights.
cudaError_t dn_flip_weights(const float* w, int co, int ci, float* wt, cudaStream_t s);
// g *= (y > 0) over c channels of n images of hw pixels.
cudaError_t dn_relu_mask(float* g, int64_t g_ns, const float* y, int64_t y_ns, int c, int n, int hw,
                         cudaStream_t s);
// 2x2 average pool of an h x w input (h, w even) and its adjoint
// (din = dout / 4 on each of the 4 pixels, added to din if accumulate).
cudaError_t dn_pool2(const float* in, int64_t in_ns, float* out, int64_t out_ns, int c, int n, int h,
                     int w, cudaStream_t s);
cudaError_t dn_pool2_bwd(const float* dout, int64_t dout_ns, float* din, int64_t din_ns, int c, int n,
                         int h, int w, bool accumulate, cudaStream_t s);
// Nearest 2x upsample of an h x w input and its adjoint (din = sum of the
// 4 output pixels).
cudaError_t dn_up2(const float* in, int64_t in_ns, float* out, int64_t out_ns, int c, int n, int h,
                   int w, cudaStream_t s);
cudaError_t dn_up2_bwd(const float* dout, int64_t dout_ns, float* din, int64_t din_ns, int c, int n,
                       int h, int w, cudaStream_t s);
// y += x over c channels of n images of hw pixels.
cudaError_t dn_add(float* y, int64_t y_ns, const float* x, int64_t x_ns, int c, int n, int hw,
                   cudaStream_t s);
// grad = 2 (pred - target) / count; *loss_sum += sum (pred - target)^2.
cudaError_t dn_mse(const float* pred, const float* target, int64_t count, float* grad,
                   float* loss_sum, cudaStream_t s);
// One Adam step (bias-corrected, step >= 1) over count parameters.
cudaError_t dn_adam(float* p, const float* g, float* m, float* v, int64_t count, float lr, float b1,
                    float b2, float eps, int step, cudaStream_t s);

}  // namespace pyr3
