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

// visualize uniforms (src/visualize.ts:178-204), curves/HSL off.
struct TonemapParams {
  uint32_t width, height, oversample, fwidth;
  float k1, k2, gamma, vibrancy, highpow, linrange;
  float bg[3];
  int transparent;
};

cudaError_t build_kw_table(const float* knorm, float* tab, cudaStream_t s);
size_t kw_table_floats();
cudaError_t launch_density(const uint32_t* hist, float* filtered, const DeParams& p,
                           const float* knorm, const float* tab, cudaStream_t s);
cudaError_t launch_tonemap(const uint32_t* hist_u32, const float* filtered, const TonemapParams& p,
                           const float* kern, void* out, bool rgba8, cudaStream_t s);

}  // namespace pyr3
