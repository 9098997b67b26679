// Density estimation + tonemap passes (device side in passes.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pyr3 {

constexpr int kMaxTaps = 17;  // src/spatial-filter.ts:195-196

// DE uniforms (src/density.ts:147-163): radii already scaled to super-res
// (max_rad * oversample + 1), k1/k2 from the calibration.
struct DeParams {
  uint32_t width, height;  // super-res
  float max_rad, min_rad, curve, k1, k2;
  int R;                   // ceil(clamp(max_rad, 0, 256))
};

// visualize uniforms (src/visualize.ts:178-204).
struct TonemapParams {
  uint32_t width, height, oversample, fwidth;
  float k1, k2, gamma, vibrancy, highpow, linrange;
  float bg[3];
  int transparent;
  uint32_t curves_active;  // channel-curves mask: composite 1, r 2, g 4, b 8, luma 16
  uint32_t hsl_active;
  float hsl_hue, hsl_sat, hsl_light;  // degrees, multiplier, addend
};

// Output kinds of a present (the PYR3_OUT_* values of the C-ABI):
//   rgba8      W x H x 4 u8, the rgba8unorm display texture;
//   rgba32f    W x H x 4 f32, the fragment value;
//   rgba16f    W x H x 4 binary16 (nearest even), the rgba16float texture;
//   png16      W x H x 4 u16, displayHalfToPng16 of the rgba16float value
//              (src/gpu-readback.ts:106-115);
//   exr display W x H x 4 f32, displayHalfToLinearExr of it
//              (src/gpu-readback.ts:83-104): sRGB-to-linear RGB, alpha as is.
enum OutKind { kOutRgba8 = 0, kOutRgba32f = 1, kOutRgba16f = 2, kOutPng16 = 3, kOutExrDisplay = 4 };
// Bytes per pixel of an output kind (0 for an unknown kind).
size_t out_bytes_per_pixel(int out_kind);

cudaError_t build_kw_table(const float* knorm, float* tab, cudaStream_t s);
size_t kw_table_floats();
// Density estimation of a super-res histogram (16-byte aligned) into
// filtered.  Kernel radii up to kDensityTmaMaxR run the TMA-staged tile
// kernel, larger ones the streaming kernel.  fault (nullable): bit 3 is set
// if a tile's copy did not land within its bounded wait (that tile is NaN).
constexpr int kDensityTmaMaxR = 31;
cudaError_t launch_density(const uint32_t* hist, float* filtered, const DeParams& p,
                           const float* knorm, const float* tab, unsigned long long* fault, cudaStream_t s);
// curves: 5 x 256 f32 LUT on the device (read only when p.curves_active != 0).
// Interior tiles of the shared-memory tile pass arrive by TMA tensor copies
// (16-byte aligned source); fault (nullable): bit 4 is set if a tile's copy
// did not land within its bounded wait (that tile's pixels are NaN).
cudaError_t launch_tonemap(const uint32_t* hist_u32, const float* filtered, const TonemapParams& p,
                           const float* kern, const float* curves, void* out, int out_kind,
                           unsigned long long* fault, cudaStream_t s);
// An rgba32f fragment-value image (16-byte aligned) written as another
// output kind, with the same per-pixel steps as the tonemap's store.
cudaError_t launch_convert_display(const float* in, uint64_t pixels, int out_kind, void* out, int sms,
                                   cudaStream_t s);

// Random-splat atomic rate: `splats` deposits of 4 saturating u32 atomics
// (the chaos kernel's scatter) into uniformly random cells of `cells`.
cudaError_t launch_splat_rate(uint32_t* cells, uint64_t n_cells, uint64_t splats, int sms, cudaStream_t s);
// histogramToLinearRgba (src/export-linear.ts:24-47): box-collapse of each
// oversample x oversample block in f64, scaled by k1 * k2 / oversample^2;
// coverage (alpha) clamped to [0, 1].  out = width x height x RGBA f32.
cudaError_t launch_linear_export(const uint32_t* hist, uint32_t width, uint32_t height,
                                 uint32_t oversample, double k1, double k2, float* out,
                                 cudaStream_t s);

// Luminance sum of an RGBA image, the numerator of computeMeanLuminance /
// computeMeanLuminanceHalf (src/auto-exposure.ts:70-97), as an exact
// integer added to *sum (which the caller zeroes):
//   rgba8  : sum over pixels of R + G + B (bytes; alpha ignored);
//   rgba32f: each of R, G, B rounded to binary16 (nearest even, the
//            rgba16float texture the reference measures), non-finite -> 0,
//            clamped to [0, 1], in units of 2^-24 (exact: every binary16
//            value in [0, 1] is a multiple of 2^-24);
//   rgba16f: the same from the binary16 values themselves.
// img must be 16-byte aligned.  The sum does not depend on the order of the
// additions, so it is the same on every run.
cudaError_t launch_luma_sum(const void* img, uint64_t pixels, int kind, unsigned long long* sum,
                            int sms, cudaStream_t s);

}  // namespace pyr3
