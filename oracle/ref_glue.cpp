// C entry points around the reference's own WGSL shaders compiled for the
// CPU by oracle/wgsl2cpp.py.  TEST INFRASTRUCTURE ONLY: this is the
// "reference" oracle (oracle/_ref/libpyr3_ref.so) used to validate the C
// restatement (oracle/oracle.c), to check the CUDA variations per point,
// and as the timed CPU baseline.  The product never links it.
//
// The translated shader namespaces (chaos, density, visualize_u32,
// visualize_f32) keep the reference's binding names; this file binds the
// module-scope storage/uniform variables and calls the entry points:
//   chaos_main     src/shaders/chaos.wgsl:8269
//   apply_variation chaos.wgsl:7731, dc_color_for chaos.wgsl:8192
//   density_main   src/shaders/density.wgsl:51
//   fs             src/shaders/visualize_u32.wgsl:147 / visualize_f32.wgsl:162
#include "../wgsl_rt.hpp"

#include <algorithm>
#include <thread>
#include <vector>

#include "chaos.cpp"  // generated into oracle/_ref/
#include "density.cpp"
#include "visualize_f32.cpp"
#include "visualize_u32.cpp"

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

static_assert(sizeof(chaos::Uniforms) == 124, "chaos uniforms layout");
static_assert(sizeof(chaos::Xform) == 464, "xform layout");
static_assert(sizeof(chaos::IsaacState) == 144, "isaac layout");

namespace {
constexpr uint32_t GRAIN = 16384;
constexpr uint32_t MAX_XFORMS = 128;

void bind_chaos(const uint32_t *uniforms31, const float *xforms, const float *palette,
                const uint32_t *distrib_full, uint32_t *isaac, uint32_t *hist, uint32_t *idx_sum,
                float *trace) {
  std::memcpy(&chaos::u, uniforms31, sizeof(chaos::Uniforms));
  chaos::xforms = reinterpret_cast<chaos::Xform *>(const_cast<float *>(xforms));
  chaos::palette = reinterpret_cast<wg::vec<float, 4> *>(const_cast<float *>(palette));
  chaos::xform_distrib = const_cast<uint32_t *>(distrib_full);
  chaos::isaac_states = reinterpret_cast<chaos::IsaacState *>(isaac);
  chaos::hist = hist;
  chaos::idx_sum = idx_sum;
  chaos::trace_buffer = trace;
}

// Expand the compact (n+1) x GRAIN pick table (fallback row last) into the
// reference's (MAX_XFORMS+1) x GRAIN layout (fallback row at MAX_XFORMS).
std::vector<uint32_t> expand_distrib(int n, const uint32_t *compact) {
  std::vector<uint32_t> full((size_t)(MAX_XFORMS + 1) * GRAIN, 0u);
  for (int r = 0; r < n; ++r)
    std::memcpy(&full[(size_t)r * GRAIN], compact + (size_t)r * GRAIN, GRAIN * 4);
  std::memcpy(&full[(size_t)MAX_XFORMS * GRAIN], compact + (size_t)n * GRAIN, GRAIN * 4);
  return full;
}
}  // namespace

// One apply_variation call.  isaac36 is a single ISAAC stream (walker 0),
// advanced in place by RNG-consuming variations.
REF_EXPORT void ref_eval_variation(uint32_t idx, float px, float py, float w, const float *p10,
                                   const float *a0, const float *a1, uint32_t *isaac36,
                                   float *out2) {
  chaos::isaac_states = reinterpret_cast<chaos::IsaacState *>(isaac36);
  vec2f p(px, py);
  vec4f A0(a0[0], a0[1], a0[2], a0[3]), A1(a1[0], a1[1], a1[2], a1[3]);
  vec2f r = chaos::U_apply_variation(idx, p, w, p10[0], p10[1], p10[2], p10[3], p10[4], p10[5],
                                     p10[6], p10[7], p10[8], p10[9], A0, A1, 0u);
  out2[0] = r.x;
  out2[1] = r.y;
}

// Batch of apply_variation calls on a point grid, each point with its own
// ISAAC stream (isaac = n x 36 u32, walker index = point index).
REF_EXPORT void ref_eval_variation_grid(uint32_t idx, int n, const float *pts, float w,
                                        const float *p10, const float *a0, const float *a1,
                                        uint32_t *isaac, float *out) {
  chaos::isaac_states = reinterpret_cast<chaos::IsaacState *>(isaac);
  vec4f A0(a0[0], a0[1], a0[2], a0[3]), A1(a1[0], a1[1], a1[2], a1[3]);
  for (int i = 0; i < n; ++i) {
    vec2f r = chaos::U_apply_variation(idx, vec2f(pts[2 * i], pts[2 * i + 1]), w, p10[0], p10[1],
                                       p10[2], p10[3], p10[4], p10[5], p10[6], p10[7], p10[8],
                                       p10[9], A0, A1, (uint32_t)i);
    out[2 * i] = r.x;
    out[2 * i + 1] = r.y;
  }
}

// dc_color_for (chaos.wgsl:8192): returns 1 and writes rgb when the
// variation has a direct colour.  v4 = vars[k], ve4 = vars_extra[k].
REF_EXPORT int ref_dc_color(uint32_t idx, float px, float py, const float *v4, const float *ve4,
                            float *rgb) {
  vec4f v(v4[0], v4[1], v4[2], v4[3]), ve(ve4[0], ve4[1], ve4[2], ve4[3]);
  chaos::DcColor c = chaos::U_dc_color_for(idx, vec2f(px, py), v, ve);
  rgb[0] = c.rgb.x;
  rgb[1] = c.rgb.y;
  rgb[2] = c.rgb.z;
  return c.hit ? 1 : 0;
}

// Run chaos_main for walkers [w0, w1) on `threads` host threads, all
// accumulating into one histogram with the reference's saturating CAS.
// uniforms31 = the reference's 31-slot uniform block; xforms = packed
// 464-byte slots; distrib = compact (n+1) x 16384 table (fallback last);
// isaac = walker_count x 36 u32 (walker-indexed).
REF_EXPORT void ref_chaos_run(const uint32_t *uniforms31, const float *xforms, int n_std,
                              const float *palette, const uint32_t *distrib, uint32_t *isaac,
                              uint32_t w0, uint32_t w1, uint32_t *hist, int threads) {
  std::vector<uint32_t> full = expand_distrib(n_std, distrib);
  if (threads < 1) threads = 1;
  uint32_t total = w1 > w0 ? w1 - w0 : 0;
  std::vector<std::thread> pool;
  std::vector<uint32_t> idx_dummy(16, 0);
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&, t]() {
      std::vector<float> trace(16 * 1000, 0.0f);
      std::vector<uint32_t> idx_local(1, 0);
      bind_chaos(uniforms31, xforms, palette, full.data(), isaac, hist, idx_local.data(),
                 trace.data());
      chaos::u.trace_mode = 0u;
      chaos::u.capture_index = 0u;
      for (uint32_t k = (uint32_t)t; k < total; k += (uint32_t)threads)
        chaos::U_chaos_main(vec3u(w0 + k, 0u, 0u));
    });
  }
  for (auto &th : pool) th.join();
}

// ref_chaos_run with the capture-index pass on (uniform slot 14 as given):
// every splat also adds its colour index into idx_sum (superW x superH u32).
REF_EXPORT void ref_chaos_run_capture(const uint32_t *uniforms31, const float *xforms, int n_std,
                                      const float *palette, const uint32_t *distrib, uint32_t *isaac,
                                      uint32_t w0, uint32_t w1, uint32_t *hist, uint32_t *idx_sum,
                                      int threads) {
  std::vector<uint32_t> full = expand_distrib(n_std, distrib);
  if (threads < 1) threads = 1;
  uint32_t total = w1 > w0 ? w1 - w0 : 0;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&, t]() {
      std::vector<float> trace(16 * 1000, 0.0f);
      bind_chaos(uniforms31, xforms, palette, full.data(), isaac, hist, idx_sum, trace.data());
      chaos::u.trace_mode = 0u;
      for (uint32_t k = (uint32_t)t; k < total; k += (uint32_t)threads)
        chaos::U_chaos_main(vec3u(w0 + k, 0u, 0u));
    });
  }
  for (auto &th : pool) th.join();
}

// density_main over rows [y0, y1) of a super-res histogram.
REF_EXPORT void ref_density(uint32_t width, uint32_t height, float max_rad, float min_rad,
                            float curve, float k1, float k2, const float *knorm,
                            const uint32_t *hist, float *filtered, int threads) {
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&, t]() {
      density::u.width = width;
      density::u.height = height;
      density::u.max_rad = max_rad;
      density::u.min_rad = min_rad;
      density::u.curve = curve;
      density::u.k1 = k1;
      density::u.k2 = k2;
      density::hist = const_cast<uint32_t *>(hist);
      density::filtered = filtered;
      density::kernel_norm = const_cast<float *>(knorm);
      for (uint32_t y = (uint32_t)t; y < height; y += (uint32_t)threads)
        for (uint32_t x = 0; x < width; ++x) density::U_density_main(vec3u(x, y, 0u));
    });
  }
  for (auto &th : pool) th.join();
}

// Visualize fragment shader over every output pixel.  src_u32 (DE off) or
// src_f32 (DE-filtered) is the super-res source.  out = W x H x RGBA f32.
REF_EXPORT void ref_visualize(uint32_t width, uint32_t height, float k1, float k2, float gamma,
                              float vibrancy, float highpow, float linrange, uint32_t oversample,
                              uint32_t fwidth, const float *bg3, uint32_t transparent,
                              const float *kernel1d, const uint32_t *src_u32,
                              const float *src_f32, float *out, int threads,
                              uint32_t curves_active, const float *curves5x256,
                              uint32_t hsl_active, float hsl_hue, float hsl_sat, float hsl_light) {
  if (threads < 1) threads = 1;
  std::vector<float> curves(5 * 256, 0.0f);
  if (curves5x256) curves.assign(curves5x256, curves5x256 + 5 * 256);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&, t]() {
#define SET_VIZ(NS)                                                     \
  NS::u.width = width;                                                  \
  NS::u.height = height;                                                \
  NS::u.k1 = k1;                                                        \
  NS::u.k2 = k2;                                                        \
  NS::u.gamma = gamma;                                                  \
  NS::u.vibrancy = vibrancy;                                            \
  NS::u.highpow = highpow;                                              \
  NS::u.linrange = linrange;                                            \
  NS::u.oversample = oversample;                                        \
  NS::u.fwidth = fwidth;                                                \
  NS::u.background = vec4f(bg3[0], bg3[1], bg3[2], 0.0f);               \
  NS::u.curvesActive = curves_active;                                   \
  NS::u.hslActive = hsl_active;                                         \
  NS::u.hslHue = hsl_hue;                                               \
  NS::u.hslSat = hsl_sat;                                               \
  NS::u.hslLight = hsl_light;                                           \
  NS::u.transparent = transparent;                                      \
  NS::kernel1d = const_cast<float *>(kernel1d);                         \
  NS::curves = curves.data();
      SET_VIZ(visualize_u32)
      SET_VIZ(visualize_f32)
#undef SET_VIZ
      visualize_u32::hist = const_cast<uint32_t *>(src_u32);
      visualize_f32::hist = const_cast<float *>(src_f32);
      for (uint32_t y = (uint32_t)t; y < height; y += (uint32_t)threads)
        for (uint32_t x = 0; x < width; ++x) {
          vec4f frag((float)x + 0.5f, (float)y + 0.5f, 0.0f, 1.0f);
          vec4f c = src_u32 ? visualize_u32::U_fs(frag) : visualize_f32::U_fs(frag);
          float *o = out + ((size_t)y * width + x) * 4;
          o[0] = c.x;
          o[1] = c.y;
          o[2] = c.z;
          o[3] = c.w;
        }
    });
  }
  for (auto &th : pool) th.join();
}
