// The reference's chaos shader (src/shaders/chaos.wgsl + noise_perlin.wgsl)
// translated by oracle/wgsl2cpp.py with every f32 evaluated as a double.
// TEST INFRASTRUCTURE ONLY: the FP64 evaluation that the f32 variations --
// the reference's own (oracle/_ref/libpyr3_ref.so) and this library's CUDA
// ones -- are measured against.  Same operations in the same order as the
// shader, in double; ISAAC draws stay u32 (rand01 / rand_11 scale them in
// double), and a bitcast of an f32 value reads the bits of its f32 rounding.
#include "../wgsl_rt.hpp"

#include "chaos64.cpp"  // generated into oracle/_ref/

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

// apply_variation (chaos.wgsl:7731) in FP64 on a point grid, each point
// with its own ISAAC stream (isaac = n x 36 u32, walker index = point
// index); inputs are f32, outputs double.
REF_EXPORT void ref64_eval_variation_grid(uint32_t idx, int n, const float *pts, float w,
                                          const float *p10, const float *a0, const float *a1,
                                          uint32_t *isaac, double *out) {
  chaos64::isaac_states = reinterpret_cast<chaos64::IsaacState *>(isaac);
  using v2 = wg::vec<double, 2>;
  using v4 = wg::vec<double, 4>;
  v4 A0(a0[0], a0[1], a0[2], a0[3]), A1(a1[0], a1[1], a1[2], a1[3]);
  for (int i = 0; i < n; ++i) {
    v2 r = chaos64::U_apply_variation(idx, v2(pts[2 * i], pts[2 * i + 1]), w, p10[0], p10[1],
                                      p10[2], p10[3], p10[4], p10[5], p10[6], p10[7], p10[8],
                                      p10[9], A0, A1, (uint32_t)i);
    out[2 * i] = r.x;
    out[2 * i + 1] = r.y;
  }
}
