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

cudaError_t build_kw_table(const float* knorm, float* tab, cudaStream_t s);
size_t kw_table_floats();
cudaError_t launch_density(const uint32_t* hist, float* filtered, const DeParams& p,
                           const float* knorm, const float* tab, cudaStream_t s);
// curves: 5 x 256 f32 LUT on the device (read only when p.curves_active != 0).
cudaError_t launch_tonemap(const uint32_t* hist_u32, const float* filtered, const TonemapParams& p,
                           const float* kern, const float* curves, void* out, bool rgba8,
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
//            value in [0, 1] is a multiple of 2^-24).
// img must be 16-byte aligned.  The sum does not depend on the order of the
// additions, so it is the same on every run.
cudaError_t launch_luma_sum(const void* img, uint64_t pixels, bool rgba8, unsigned long long* sum,
                            int sms, cudaStream_t s);

}  // namespace pyr3
