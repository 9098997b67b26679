// Variation evaluator (NVRTC template): one thread per point, each point
// with its own ISAAC stream given in the reference layout
// [cnt, a, b, c, mem[16], rsl[16]] and written back after the call.  The
// generator defines EVAL_VAR (and EVAL_DC for direct-colour variations).
#pragma once
#define EWPB 128

extern "C" __global__ void __launch_bounds__(EWPB)
eval_kernel(u32 n, const float2* __restrict__ pts, float w, const float* __restrict__ prm,
            float4 a0, float4 a1, u32* isaac, float2* out) {
  __shared__ u32 st[36 * EWPB];
  const u32 t = threadIdx.x;
  const u64 i = (u64)blockIdx.x * EWPB + t;
  if (i >= n) return;
  for (int k = 0; k < 36; ++k) st[k * EWPB + t] = isaac[i * 36 + k];
  Ctx c;
  c.rng = Rng{st + t, EWPB};
  c.a0 = a0;
  c.a1 = a1;
  float P[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) P[k] = prm[k];
  out[i] = EVAL_VAR(pts[i], w, P, c);
  for (int k = 0; k < 36; ++k) isaac[i * 36 + k] = st[k * EWPB + t];
}

#ifdef EVAL_DC
extern "C" __global__ void dc_kernel(u32 n, const float2* __restrict__ pts,
                                     const float* __restrict__ prm, float* out_rgb) {
  const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float P[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) P[k] = prm[k];
  float3 c = EVAL_DC(pts[i], P);
  out_rgb[i * 3 + 0] = c.x;
  out_rgb[i * 3 + 1] = c.y;
  out_rgb[i * 3 + 2] = c.z;
}
#endif
