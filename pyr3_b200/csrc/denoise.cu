// Denoiser kernels (see denoise.h).  f32 on the CUDA cores: the
// convolution stages a 16 x 16 output tile (+1 halo) of 4 input channels and
// the matching 8 x 4 x 9 weights in shared memory per step; each thread
// accumulates 8 output channels of one pixel.
#include "denoise.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

namespace pyr3 {
namespace {

constexpr int TS = 16;    // output tile edge
constexpr int CO_B = 8;   // output channels per block
constexpr int CI_B = 4;   // input channels staged per step
constexpr int kWgChunks = 128;  // pixel chunks of the weight gradient (partials added in a fixed order)

__global__ void __launch_bounds__(256)
k_conv3x3(const float* __restrict__ in, int64_t in_ns, int ci_n, float* __restrict__ out,
          int64_t out_ns, int co_n, int H, int W, const float* __restrict__ wt,
          const float* __restrict__ bias, int relu) {
  __shared__ float tile[CI_B][TS + 2][TS + 3];
  __shared__ float ws[CI_B][9][CO_B];
  const int tx = threadIdx.x & (TS - 1), ty = threadIdx.x / TS;
  const int x0 = blockIdx.x * TS, y0 = blockIdx.y * TS;
  const int groups = (co_n + CO_B - 1) / CO_B;
  const int n = blockIdx.z / groups, co0 = (blockIdx.z % groups) * CO_B;
  const int64_t hw = (int64_t)H * W;
  const float* inn = in + n * in_ns;
  float acc[CO_B];
#pragma unroll
  for (int j = 0; j < CO_B; ++j) acc[j] = 0.0f;
  for (int c0 = 0; c0 < ci_n; c0 += CI_B) {
    for (int i = threadIdx.x; i < CI_B * (TS + 2) * (TS + 2); i += 256) {
      const int c = i / ((TS + 2) * (TS + 2)), r = i % ((TS + 2) * (TS + 2));
      const int yy = r / (TS + 2), xx = r % (TS + 2);
      const int gy = y0 + yy - 1, gx = x0 + xx - 1;
      float v = 0.0f;
      if (c0 + c < ci_n && gy >= 0 && gy < H && gx >= 0 && gx < W)
        v = inn[(c0 + c) * hw + (int64_t)gy * W + gx];
      tile[c][yy][xx] = v;
    }
    for (int i = threadIdx.x; i < CO_B * CI_B * 9; i += 256) {
      const int j = i / (CI_B * 9), r = i % (CI_B * 9), c = r / 9, k = r % 9;
      float v = 0.0f;
      if (co0 + j < co_n && c0 + c < ci_n) v = wt[((int64_t)(co0 + j) * ci_n + c0 + c) * 9 + k];
      ws[c][k][j] = v;
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < CI_B; ++c) {
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const float v = tile[c][ty + k / 3][tx + k % 3];
#pragma unroll
        for (int j = 0; j < CO_B; ++j) acc[j] = fmaf(ws[c][k][j], v, acc[j]);
      }
    }
    __syncthreads();
  }
  const int x = x0 + tx, y = y0 + ty;
  if (x >= W || y >= H) return;
#pragma unroll
  for (int j = 0; j < CO_B; ++j) {
    if (co0 + j >= co_n) break;
    float r = acc[j] + (bias ? bias[co0 + j] : 0.0f);
    if (relu) r = fmaxf(r, 0.0f);
    out[n * out_ns + (co0 + j) * hw + (int64_t)y * W + x] = r;
  }
}

// Weight and bias gradient, split over pixels: block (ci group of 4, co
// group of 2, chunk s) accumulates the 2 x 4 x 9 taps (and, for the first
// ci group, the 2 bias sums) over pixel chunk s of all images into
// part[s]; k_wgrad_reduce adds the kWgChunks partials in a fixed order.
constexpr int WG_CI = 4, WG_CO = 2;

__global__ void __launch_bounds__(256)
k_wgrad_part(const float* __restrict__ in, int64_t in_ns, int ci_n, const float* __restrict__ dout,
             int64_t dout_ns, int co_n, int n_img, int H, int W, float* __restrict__ part,
             float* __restrict__ part_b) {
  const int ci0 = blockIdx.x * WG_CI, co0 = blockIdx.y * WG_CO, s = blockIdx.z;
  const int64_t hw = (int64_t)H * W, P = hw * n_img;
  const int64_t p0 = P * s / kWgChunks, p1 = P * (s + 1) / kWgChunks;
  float a[WG_CO][WG_CI][9], b[WG_CO];
#pragma unroll
  for (int j = 0; j < WG_CO; ++j) {
    b[j] = 0.0f;
#pragma unroll
    for (int c = 0; c < WG_CI; ++c)
#pragma unroll
      for (int k = 0; k < 9; ++k) a[j][c][k] = 0.0f;
  }
  for (int64_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
    const int64_t n = p / hw, r = p % hw;
    const int y = (int)(r / W), x = (int)(r % W);
    float g[WG_CO];
#pragma unroll
    for (int j = 0; j < WG_CO; ++j) g[j] = co0 + j < co_n ? dout[n * dout_ns + (co0 + j) * hw + r] : 0.0f;
    if (g[0] == 0.0f && g[1] == 0.0f) continue;  // ReLU-masked gradients are often zero
#pragma unroll
    for (int j = 0; j < WG_CO; ++j) b[j] += g[j];
#pragma unroll
    for (int c = 0; c < WG_CI; ++c) {
      if (ci0 + c >= ci_n) break;
      const float* ip = in + n * in_ns + (ci0 + c) * hw;
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const int gy = y + k / 3 - 1, gx = x + k % 3 - 1;
        const float v = (gy >= 0 && gy < H && gx >= 0 && gx < W) ? ip[(int64_t)gy * W + gx] : 0.0f;
#pragma unroll
        for (int j = 0; j < WG_CO; ++j) a[j][c][k] = fmaf(g[j], v, a[j][c][k]);
      }
    }
  }
  // Block sums: warp shuffles, then one value per warp through shared memory.
  constexpr int NV = WG_CO * WG_CI * 9 + WG_CO;
  __shared__ float red[NV][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    float x = v < WG_CO * WG_CI * 9 ? a[v / (WG_CI * 9)][(v / 9) % WG_CI][v % 9] : b[v - WG_CO * WG_CI * 9];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[v][warp] = x;
  }
  __syncthreads();
  for (int v = threadIdx.x; v < NV; v += blockDim.x) {
    float x = 0.0f;
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) x += red[v][j];
    if (v < WG_CO * WG_CI * 9) {
      const int j = v / (WG_CI * 9), c = (v / 9) % WG_CI, k = v % 9;
      if (co0 + j < co_n && ci0 + c < ci_n)
        part[(((int64_t)s * co_n + co0 + j) * ci_n + ci0 + c) * 9 + k] = x;
    } else if (blockIdx.x == 0) {
      const int j = v - WG_CO * WG_CI * 9;
      if (co0 + j < co_n) part_b[(int64_t)s * co_n + co0 + j] = x;
    }
  }
}

__global__ void k_wgrad_reduce(const float* __restrict__ part, int64_t per, int parts, float* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= per) return;
  float x = 0.0f;
  for (int s = 0; s < parts; ++s) x += part[s * per + i];
  out[i] = x;
}

__global__ void k_flip(const float* __restrict__ w, int co_n, int ci_n, float* __restrict__ wt) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)co_n * ci_n * 9) return;
  const int k = (int)(i % 9);
  const int64_t r = i / 9;
  const int ci = (int)(r % ci_n), co = (int)(r / ci_n);
  wt[((int64_t)ci * co_n + co) * 9 + (8 - k)] = w[i];
}

// Element r of c channels x hw pixels of image n lives at n * ns + r; the
// grid's y is the image.
__global__ void k_relu_mask(float* g, int64_t g_ns, const float* __restrict__ y, int64_t y_ns, int64_t per) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
  if (r >= per) return;
  if (!(y[n * y_ns + r] > 0.0f)) g[n * g_ns + r] = 0.0f;
}

__global__ void k_add(float* y, int64_t y_ns, const float* __restrict__ x, int64_t x_ns, int64_t per) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, n = blockIdx.y;
  if (r >= per) return;
  y[n * y_ns + r] += x[n * x_ns + r];
}

// One thread per output pixel of the half-size plane.
__global__ void k_pool2(const float* __restrict__ in, int64_t in_ns, float* out, int64_t out_ns, int c_n,
                        int n_img, int H, int W) {
  const int h2 = H / 2, w2 = W / 2;
  const int64_t per = (int64_t)c_n * h2 * w2;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= per * n_img) return;
  const int64_t n = i / per, r = i % per;
  const int64_t c = r / ((int64_t)h2 * w2), q = r % ((int64_t)h2 * w2);
  const int y = (int)(q / w2), x = (int)(q % w2);
  const float* p = in + n * in_ns + c * H * W + (int64_t)(2 * y) * W + 2 * x;
  out[n * out_ns + r] = 0.25f * ((p[0] + p[1]) + (p[W] + p[W + 1]));
}

__global__ void k_pool2_bwd(const float* __restrict__ dout, int64_t dout_ns, float* din, int64_t din_ns,
                            int c_n, int n_img, int H, int W, int accumulate) {
  const int h2 = H / 2, w2 = W / 2;
  const int64_t per = (int64_t)c_n * h2 * w2;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= per * n_img) return;
  const int64_t n = i / per, r = i % per;
  const int64_t c = r / ((int64_t)h2 * w2), q = r % ((int64_t)h2 * w2);
  const int y = (int)(q / w2), x = (int)(q % w2);
  const float g = 0.25f * dout[n * dout_ns + r];
  float* p = din + n * din_ns + c * H * W + (int64_t)(2 * y) * W + 2 * x;
  if (accumulate) {
    p[0] += g; p[1] += g; p[W] += g; p[W + 1] += g;
  } else {
    p[0] = g; p[1] = g; p[W] = g; p[W + 1] = g;
  }
}

// in is h x w; one thread per input pixel writes its 2 x 2 block.
__global__ void k_up2(const float* __restrict__ in, int64_t in_ns, float* out, int64_t out_ns, int c_n,
                      int n_img, int H, int W) {
  const int64_t per = (int64_t)c_n * H * W;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= per * n_img) return;
  const int64_t n = i / per, r = i % per;
  const int64_t c = r / ((int64_t)H * W), q = r % ((int64_t)H * W);
  const int y = (int)(q / W), x = (int)(q % W);
  const float v = in[n * in_ns + r];
  float* p = out + n * out_ns + c * 4 * H * W + (int64_t)(2 * y) * (2 * W) + 2 * x;
  p[0] = v; p[1] = v; p[2 * W] = v; p[2 * W + 1] = v;
}

__global__ void k_up2_bwd(const float* __restrict__ dout, int64_t dout_ns, float* din, int64_t din_ns,
                          int c_n, int n_img, int H, int W) {
  const int64_t per = (int64_t)c_n * H * W;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= per * n_img) return;
  const int64_t n = i / per, r = i % per;
  const int64_t c = r / ((int64_t)H * W), q = r % ((int64_t)H * W);
  const int y = (int)(q / W), x = (int)(q % W);
  const float* p = dout + n * dout_ns + c * 4 * H * W + (int64_t)(2 * y) * (2 * W) + 2 * x;
  din[n * din_ns + r] = (p[0] + p[1]) + (p[2 * W] + p[2 * W + 1]);
}

__global__ void __launch_bounds__(256)
k_mse(const float* __restrict__ pred, const float* __restrict__ tgt, int64_t count, float* grad,
      float* loss_sum) {
  float a = 0.0f;
  const float sc = 2.0f / (float)count;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float d = pred[i] - tgt[i];
    grad[i] = sc * d;
    a = fmaf(d, d, a);
  }
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss_sum, a);
}

__global__ void k_adam(float* p, const float* __restrict__ g, float* m, float* v, int64_t count,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

unsigned blocks_for(int64_t n, int bs = 256) { return (unsigned)((n + bs - 1) / bs); }

// ---- 3x3 convolution on the tensor cores (tcgen05, bf16 x bf16 -> f32)
// Implicit GEMM without im2col.  Index the zero-padded input by position
// q = (y + 1) * P + (x + 1), P = W + 2: output q reads input q + d for tap
// (ky, kx), d = (ky - 1) * P + (kx - 1) -- the same shift for every pixel.
// A CTA owns T tiles of 128 consecutive output positions (M = 128 each;
// positions in the padding columns are computed and dropped; T <= 4, one
// TMEM accumulator per tile) and stages the padded input rows they need,
// R = 128 T + 2 (P + 1), once -- the tap window of the tiles' rows above and
// below is shared by all T tiles: plane g holds channels 8g..8g+7
// as one 16-byte bf16 row per position, so the operand of tap t and K step
// s (channels 16s..16s+15) is planes 2s and 2s+1 read from row P + 1 + d_t:
// a no-swizzle K-major descriptor with contiguous rows (SBO = 16 B x 8) and
// the next plane at LBO = 16 R bytes.  The weights (all output channels,
// N = NP padded to 16) are staged beside the input in the usual canonical
// layout, once for all T tiles, TG taps at a time (all nine where shared
// memory allows); one thread issues the group's MMAs of every tile into
// its TMEM accumulator and commits them to an mbarrier that every thread
// waits on (bounded).  Each warp reads its 32 rows back (tcgen05.ld), adds
// the bias, applies ReLU and stores the interior pixels in f32.
constexpr uint32_t TC_WAIT_LIMIT = 1u << 24;
constexpr int TC_MAX_SMEM = 200 * 1024;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  // start >> 4, leading / stride byte offsets >> 4, descriptor version 1, no swizzle
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// Dynamic shared memory of the tensor-core convolution (bytes), T tiles:
// the staged input planes and the weights of TG taps.
__host__ __device__ inline size_t tc_smem_bytes(int ci, int w, int np, int T, int TG) {
  const size_t R = 128 * (size_t)T + 2 * (size_t)(w + 3);
  const size_t G = 2 * (size_t)((ci + 15) / 16);
  return G * R * 16 + (size_t)TG * (G / 2) * (size_t)np * 32;
}

template <int NP>
__global__ void __launch_bounds__(128)
k_conv3x3_tc(const float* __restrict__ in, int64_t in_ns, int ci_n, float* __restrict__ out, int64_t out_ns,
             int co_n, int H, int W, const float* __restrict__ wt, const float* __restrict__ bias, int relu,
             int T, int TG) {
  constexpr uint32_t NCOL = NP <= 32 ? 32 : (NP <= 64 ? 64 : 128);
  // TMEM columns: one NCOL accumulator per tile, allocated as a power of two.
  const uint32_t ncols = (uint32_t)T * NCOL <= 32u ? 32u : ((uint32_t)T * NCOL <= 64u ? 64u :
                         ((uint32_t)T * NCOL <= 128u ? 128u : ((uint32_t)T * NCOL <= 256u ? 256u : 512u)));
  extern __shared__ __align__(1024) unsigned char smem[];
  const int P = W + 2, R = 128 * T + 2 * (P + 1), G = 2 * ((ci_n + 15) / 16), S = G / 2;
  uint4* sa = reinterpret_cast<uint4*>(smem);  // G planes x R rows of 16 B
  uint4* sb = sa + (size_t)G * R;               // TG taps x S K steps x (NP / 8) x 2 core matrices x 8 rows
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int n = blockIdx.y;
  const int q0 = P + 1 + blockIdx.x * 128 * T;  // first output position of the CTA's first tile
  const int qa = q0 - (P + 1);              // position of staged row 0
  const int64_t hw = (int64_t)H * W;
  const float* inn = in + n * in_ns;
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n"
                 "fence.mbarrier_init.release.cluster;" ::"r"(smem_addr(&bar)) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                 "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // padded input rows: plane g, row r = position qa + r, 8 channels as bf16
  for (int i = t; i < G * R; i += 128) {
    const int g = i / R, r = i - g * R;
    const int q = qa + r, yy = q / P - 1, xx = q % P - 1;
    float v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = 0.0f;
    if (yy >= 0 && yy < H && xx >= 0 && xx < W) {
      const float* ip = inn + (int64_t)yy * W + xx;
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (g * 8 + j < ci_n) v[j] = ip[(int64_t)(g * 8 + j) * hw];
    }
    sa[i] = make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NP >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  const uint32_t lbo_a = (uint32_t)R * 16u;
  const int per_tap = S * NP * 2;  // uint4 rows of one tap's weights
  // Taps in groups of TG (all nine where shared memory allows): the group's
  // weights B[co][16 s + kk] = w[co][16 s + kk][tap] are staged, one thread
  // issues the group's MMAs of every tile into its TMEM accumulator and
  // commits them to an mbarrier that every thread waits on (bounded) before
  // the next group's weights overwrite these.
  for (int tap0 = 0, ph = 0; tap0 < 9; tap0 += TG, ++ph) {
    const int ntap = min(TG, 9 - tap0);
    for (int idx = t; idx < ntap * per_tap; idx += 128) {
      const int k = idx / per_tap, r0 = idx - k * per_tap, tap = tap0 + k;
      const int s = r0 / (NP * 2), rem = r0 - s * NP * 2, co = rem >> 1, h = rem & 1;
      float v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int ci = s * 16 + h * 8 + j;
        v[j] = (co < co_n && ci < ci_n) ? wt[((int64_t)co * ci_n + ci) * 9 + tap] : 0.0f;
      }
      sb[k * per_tap + (s * (NP / 4) + (co >> 3) * 2 + h) * 8 + (co & 7)] =
          make_uint4(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7]));
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int k = 0; k < ntap; ++k) {
        const int tap = tap0 + k;
        const int row0 = (P + 1) + (tap / 3 - 1) * P + (tap % 3 - 1);
        for (int m = 0; m < T; ++m) {  // tile m: rows 128 m.. of the window, accumulator columns m NCOL..
          for (int s = 0; s < S; ++s) {
            const uint64_t da = umma_desc(smem_addr(sa + (size_t)(2 * s) * R + row0 + 128 * m), lbo_a, 128u);
            const uint64_t db = umma_desc(smem_addr(sb + (size_t)k * per_tap + (size_t)s * NP * 2), 128u, 256u);
            const uint32_t acc = (tap > 0 || s > 0) ? 1u : 0u;
            asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                         " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                         ::"r"(tmem + (uint32_t)m * NCOL), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   ::"r"(smem_addr(&bar)) : "memory");
    }
    uint32_t done = 0;
    for (uint32_t it = 0; it < TC_WAIT_LIMIT && !done; ++it)
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                   : "=r"(done) : "r"(smem_addr(&bar)), "r"((uint32_t)(ph & 1)) : "memory");
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  // epilogue: TMEM row i of accumulator m = output position q0 + 128 m + i
#pragma unroll 1
  for (int m = 0; m < T; ++m) {
    const int q = q0 + 128 * m + warp * 32 + lane, oy = q / P - 1, ox = q % P - 1;
    const bool inside = oy >= 0 && oy < H && ox >= 0 && ox < W;
#pragma unroll 1
    for (int c0 = 0; c0 < NP; c0 += 8) {
      uint32_t v[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(m * NCOL + c0)));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (inside) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int co = c0 + j;
          if (co < co_n) {
            float x = __uint_as_float(v[j]) + (bias ? bias[co] : 0.0f);
            if (relu) x = fmaxf(x, 0.0f);
            out[n * out_ns + co * hw + (int64_t)oy * W + ox] = x;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// ---- weight gradient on the tensor cores
// dW[co][ci][tap] = sum over positions q of dout[q][co] * in[q + d_tap][ci],
// q over the zero-padded grid (P = W + 2), so for each tap it is a GEMM
// with M = output channels (padded to 128), N = input channels (padded to
// NP), K = positions.  CTA (chunk c, image n, tap) reduces its chunk of
// positions in steps of 64: the 128 threads stage dout rows (A, zero at
// padding positions) and the tap-shifted input rows (B) as bf16 in the
// canonical K-major layout, one thread issues four K = 16 MMAs into TMEM
// and commits to the mbarrier (bounded waits); the epilogue writes the
// chunk's partial dW[co][ci][tap] to part[c * n_img + n], which
// k_wgrad_reduce adds in a fixed order.
constexpr int WT_KC = 64;

template <int NP>
__global__ void __launch_bounds__(128)
k_wgrad_tc(const float* __restrict__ in, int64_t in_ns, int ci_n, const float* __restrict__ dout,
           int64_t dout_ns, int co_n, int H, int W, int chunk, float* __restrict__ part) {
  constexpr uint32_t NCOL = NP <= 32 ? 32 : (NP <= 64 ? 64 : 128);
  extern __shared__ __align__(1024) unsigned char smem[];
  uint4* sa = reinterpret_cast<uint4*>(smem);  // 4 K steps x 128 rows x 2 halves x 16 B
  uint4* sb = sa + 4 * 128 * 2;                 // 4 K steps x NP rows x 2 halves x 16 B
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int c = blockIdx.x, n = blockIdx.y, tap = blockIdx.z;
  const int P = W + 2;
  const int d = (tap / 3 - 1) * P + (tap % 3 - 1);
  const int q_begin = P + 1 + c * chunk;
  const int q_end = min(q_begin + chunk, H * P + W + 1);  // past the last interior position
  const int64_t hw = (int64_t)H * W;
  const float* dn = dout + n * dout_ns;
  const float* ip = in + n * in_ns;
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n"
                 "fence.mbarrier_init.release.cluster;" ::"r"(smem_addr(&bar)) : "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_base)),
                 "r"(NCOL) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NP >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  // A rows co_n..127 (output channels past the layer's) are zero for every step.
  for (int idx = co_n * (WT_KC / 8) + t; idx < 128 * (WT_KC / 8); idx += 128) {
    const int co = idx >> 3, g = idx & 7, s = g >> 1, h = g & 1;
    sa[(s * 32 + (co >> 3) * 2 + h) * 8 + (co & 7)] = make_uint4(0u, 0u, 0u, 0u);
  }
  int phase = 0;
  for (int qs = q_begin; qs < q_end; qs += WT_KC, ++phase) {
    // A rows (output channel co: dout, zero at padding positions and past
    // the chunk) and B rows (input channel ci: the input at the position
    // shifted by the tap), as bf16 in the operands' 16-byte rows of 8
    // positions.  Each thread stages one position of the step, p = t mod 64,
    // for every second channel, so the lanes of a warp read 32 consecutive
    // positions of one channel: one coalesced request per load.  A rows past
    // co_n stay zero (written once, above).
    {
      const int p = t & (WT_KC - 1);
      const int q = qs + p, qi = q + d;  // qi >= 0: q >= P + 1, d >= -(P + 1)
      const int yy = q / P, xx = q - yy * P;
      const int yi = qi / P, xi = qi - yi * P;
      const bool in_a = q < q_end && yy >= 1 && yy <= H && xx >= 1 && xx <= W;
      const bool in_b = q < q_end && yi >= 1 && yi <= H && xi >= 1 && xi <= W;
      const int64_t off_a = (int64_t)(yy - 1) * W + (xx - 1), off_b = (int64_t)(yi - 1) * W + (xi - 1);
      const int g = p >> 3, s = g >> 1, h = g & 1, e = p & 7;
      unsigned short* sa16 = reinterpret_cast<unsigned short*>(sa);
      unsigned short* sb16 = reinterpret_cast<unsigned short*>(sb);
      for (int co = t / WT_KC; co < co_n; co += 128 / WT_KC) {
        const float v = in_a ? dn[co * hw + off_a] : 0.0f;
        sa16[((s * 32 + (co >> 3) * 2 + h) * 8 + (co & 7)) * 8 + e] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
      }
      for (int ci = t / WT_KC; ci < NP; ci += 128 / WT_KC) {
        const float v = (in_b && ci < ci_n) ? ip[ci * hw + off_b] : 0.0f;
        sb16[((s * (NP / 4) + (ci >> 3) * 2 + h) * 8 + (ci & 7)) * 8 + e] = __bfloat16_as_ushort(__float2bfloat16_rn(v));
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int s = 0; s < 4; ++s) {
        const uint64_t da = umma_desc(smem_addr(sa + (size_t)s * 128 * 2), 128u, 256u);
        const uint64_t db = umma_desc(smem_addr(sb + (size_t)s * NP * 2), 128u, 256u);
        const uint32_t acc = (phase > 0 || s > 0) ? 1u : 0u;
        asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                     " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                     ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   ::"r"(smem_addr(&bar)) : "memory");
    }
    uint32_t done = 0;
    for (uint32_t it = 0; it < TC_WAIT_LIMIT && !done; ++it)
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                   : "=r"(done) : "r"(smem_addr(&bar)), "r"((uint32_t)(phase & 1)) : "memory");
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  // epilogue: TMEM row co, column ci (a chunk without positions leaves zeros)
  const int co = warp * 32 + lane;
  float* pp = part + (int64_t)(c * gridDim.y + n) * co_n * ci_n * 9;
#pragma unroll 1
  for (int c0 = 0; c0 < NP; c0 += 8) {
    uint32_t v[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    if (co < co_n) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int ci = c0 + j;
        if (ci < ci_n) pp[((int64_t)co * ci_n + ci) * 9 + tap] = phase > 0 ? __uint_as_float(v[j]) : 0.0f;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOL) : "memory");
}

__global__ void __launch_bounds__(256)
k_bias_part(const float* __restrict__ dout, int64_t dout_ns, int co_n, int n_img, int64_t hw, float* part_b) {
  // block (co, chunk s): sum of dout[co] over chunk s of all images' pixels
  const int co = blockIdx.x, s = blockIdx.y;
  const int64_t P = hw * n_img, p0 = P * s / kWgChunks, p1 = P * (s + 1) / kWgChunks;
  float a = 0.0f;
  // position p = image img, pixel off; divided once, then stepped
  int64_t p = p0 + threadIdx.x, img = p / hw, off = p - img * hw;
  for (; p < p1; p += blockDim.x) {
    a += dout[img * dout_ns + co * hw + off];
    off += blockDim.x;
    while (off >= hw) {
      off -= hw;
      ++img;
    }
  }
  __shared__ float red[8];
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    float v = 0.0f;
    for (int j = 0; j < (int)(blockDim.x >> 5); ++j) v += red[j];
    part_b[(int64_t)s * co_n + co] = v;
  }
}

}  // namespace

cudaError_t dn_conv3x3(const float* in, int64_t in_ns, int ci, float* out, int64_t out_ns, int co, int n,
                       int h, int w, const float* weight, const float* bias, bool relu, cudaStream_t s) {
  const dim3 grid((w + TS - 1) / TS, (h + TS - 1) / TS, n * ((co + CO_B - 1) / CO_B));
  k_conv3x3<<<grid, 256, 0, s>>>(in, in_ns, ci, out, out_ns, co, h, w, weight, bias, relu ? 1 : 0);
  return cudaGetLastError();
}

size_t dn_wgrad_scratch_floats(int co, int ci) { return (size_t)kWgChunks * ((size_t)co * ci * 9 + co); }

template <int NP>
cudaError_t launch_wgrad_tc(const float* in, int64_t in_ns, int ci, const float* dout, int64_t dout_ns, int co,
                            int n, int h, int w, float* part, cudaStream_t s) {
  const size_t smem = (size_t)(4 * 128 * 2 + 4 * NP * 2) * 16;
  static bool attr = false;  // per instantiation; the same limit on every device
  if (!attr) {
    const cudaError_t e = cudaFuncSetAttribute(k_wgrad_tc<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  // kWgChunks partials in all: chunks per image x images
  const int per_img = std::max(1, kWgChunks / n);
  const int64_t span = (int64_t)(h - 1) * (w + 2) + w;
  const int chunk = (int)(((span + per_img - 1) / per_img + WT_KC - 1) / WT_KC * WT_KC);
  k_wgrad_tc<NP><<<dim3(per_img, n, 9), 128, smem, s>>>(in, in_ns, ci, dout, dout_ns, co, h, w, chunk, part);
  return cudaGetLastError();
}

cudaError_t dn_conv3x3_wgrad_bf16(const float* in, int64_t in_ns, int ci, const float* dout, int64_t dout_ns,
                                  int co, int n, int h, int w, float* dw, float* db, float* scratch, cudaStream_t s) {
  if (co > 128 || n > kWgChunks) return cudaErrorInvalidValue;
  const int per_img = std::max(1, kWgChunks / n), parts = per_img * n;
  const int64_t per_w = (int64_t)co * ci * 9;
  float* part = scratch;
  float* part_b = scratch + (int64_t)kWgChunks * per_w;
  cudaError_t e;
  if (ci <= 16) e = launch_wgrad_tc<16>(in, in_ns, ci, dout, dout_ns, co, n, h, w, part, s);
  else if (ci <= 32) e = launch_wgrad_tc<32>(in, in_ns, ci, dout, dout_ns, co, n, h, w, part, s);
  else if (ci <= 48) e = launch_wgrad_tc<48>(in, in_ns, ci, dout, dout_ns, co, n, h, w, part, s);
  else if (ci <= 64) e = launch_wgrad_tc<64>(in, in_ns, ci, dout, dout_ns, co, n, h, w, part, s);
  else if (ci <= 96) e = launch_wgrad_tc<96>(in, in_ns, ci, dout, dout_ns, co, n, h, w, part, s);
  else if (ci <= 128) e = launch_wgrad_tc<128>(in, in_ns, ci, dout, dout_ns, co, n, h, w, part, s);
  else return cudaErrorInvalidValue;
  if (e != cudaSuccess) return e;
  k_wgrad_reduce<<<blocks_for(per_w), 256, 0, s>>>(part, per_w, parts, dw);
  if (db) {
    k_bias_part<<<dim3(co, kWgChunks), 256, 0, s>>>(dout, dout_ns, co, n, (int64_t)h * w, part_b);
    k_wgrad_reduce<<<blocks_for(co), 256, 0, s>>>(part_b, co, kWgChunks, db);
  }
  return cudaGetLastError();
}

template <int NP>
cudaError_t launch_tc(const float* in, int64_t in_ns, int ci, float* out, int64_t out_ns, int co, int n, int h,
                      int w, const float* weight, const float* bias, bool relu, cudaStream_t s) {
  // Tiles per CTA: up to 4 (512 TMEM columns at NP = 128) while the launch
  // keeps at least four CTAs per SM (148 SMs); fewer where the staged
  // window would not fit.  One tile per CTA for small launches, whose
  // parallelism matters more than the shared window.
  const int P = w + 2;
  const int64_t span = (int64_t)(h - 1) * P + w;  // output positions from the first to the last pixel
  const int64_t tiles = (span + 127) / 128;
  int T = (int)std::max<int64_t>(1, std::min<int64_t>({4, tiles, tiles * n / (4 * 148)}));
  // All nine taps' weights at once where they fit (one MMA burst, one
  // wait), else groups of three, else one tap at a time.
  int TG = 9;
  while (T > 1 && tc_smem_bytes(ci, w, NP, T, TG) > (size_t)TC_MAX_SMEM) --T;
  while (TG > 1 && tc_smem_bytes(ci, w, NP, T, TG) > (size_t)TC_MAX_SMEM) TG = TG > 3 ? 3 : 1;
  const size_t smem = tc_smem_bytes(ci, w, NP, T, TG);
  if (smem > (size_t)TC_MAX_SMEM) return cudaErrorInvalidValue;
  static bool attr = false;  // per instantiation; the same limit on every device
  if (!attr) {
    const cudaError_t e = cudaFuncSetAttribute(k_conv3x3_tc<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_MAX_SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  const dim3 grid((unsigned)((tiles + T - 1) / T), n);
  k_conv3x3_tc<NP><<<grid, 128, smem, s>>>(in, in_ns, ci, out, out_ns, co, h, w, weight, bias, relu ? 1 : 0, T, TG);
  return cudaGetLastError();
}

cudaError_t dn_conv3x3_bf16(const float* in, int64_t in_ns, int ci, float* out, int64_t out_ns, int co, int n,
                            int h, int w, const float* weight, const float* bias, bool relu, cudaStream_t s) {
  if (co <= 16) return launch_tc<16>(in, in_ns, ci, out, out_ns, co, n, h, w, weight, bias, relu, s);
  if (co <= 32) return launch_tc<32>(in, in_ns, ci, out, out_ns, co, n, h, w, weight, bias, relu, s);
  if (co <= 48) return launch_tc<48>(in, in_ns, ci, out, out_ns, co, n, h, w, weight, bias, relu, s);
  if (co <= 64) return launch_tc<64>(in, in_ns, ci, out, out_ns, co, n, h, w, weight, bias, relu, s);
  if (co <= 96) return launch_tc<96>(in, in_ns, ci, out, out_ns, co, n, h, w, weight, bias, relu, s);
  if (co <= 128) return launch_tc<128>(in, in_ns, ci, out, out_ns, co, n, h, w, weight, bias, relu, s);
  return cudaErrorInvalidValue;
}

cudaError_t dn_conv3x3_wgrad(const float* in, int64_t in_ns, int ci, const float* dout, int64_t dout_ns,
                             int co, int n, int h, int w, float* dw, float* db, float* scratch,
                             cudaStream_t s) {
  const int64_t per_w = (int64_t)co * ci * 9;
  float* part = scratch;
  float* part_b = scratch + kWgChunks * per_w;
  const dim3 grid((ci + WG_CI - 1) / WG_CI, (co + WG_CO - 1) / WG_CO, kWgChunks);
  k_wgrad_part<<<grid, 256, 0, s>>>(in, in_ns, ci, dout, dout_ns, co, n, h, w, part, part_b);
  k_wgrad_reduce<<<blocks_for(per_w), 256, 0, s>>>(part, per_w, kWgChunks, dw);
  if (db) k_wgrad_reduce<<<blocks_for(co), 256, 0, s>>>(part_b, co, kWgChunks, db);
  return cudaGetLastError();
}

cudaError_t dn_flip_weights(const float* w, int co, int ci, float* wt, cudaStream_t s) {
  k_flip<<<blocks_for((int64_t)co * ci * 9), 256, 0, s>>>(w, co, ci, wt);
  return cudaGetLastError();
}

cudaError_t dn_relu_mask(float* g, int64_t g_ns, const float* y, int64_t y_ns, int c, int n, int hw,
                         cudaStream_t s) {
  const int64_t per = (int64_t)c * hw;
  for (int n0 = 0; n0 < n && per > 0; n0 += 65535)  // grid y: up to 65535 images per launch
    k_relu_mask<<<dim3(blocks_for(per), std::min(65535, n - n0)), 256, 0, s>>>(g + n0 * g_ns, g_ns, y + n0 * y_ns,
                                                                             y_ns, per);
  return cudaGetLastError();
}

cudaError_t dn_add(float* y, int64_t y_ns, const float* x, int64_t x_ns, int c, int n, int hw,
                   cudaStream_t s) {
  const int64_t per = (int64_t)c * hw;
  for (int n0 = 0; n0 < n && per > 0; n0 += 65535)  // grid y: up to 65535 images per launch
    k_add<<<dim3(blocks_for(per), std::min(65535, n - n0)), 256, 0, s>>>(y + n0 * y_ns, y_ns, x + n0 * x_ns, x_ns,
                                                                       per);
  return cudaGetLastError();
}

cudaError_t dn_pool2(const float* in, int64_t in_ns, float* out, int64_t out_ns, int c, int n, int h, int w,
                     cudaStream_t s) {
  k_pool2<<<blocks_for((int64_t)c * (h / 2) * (w / 2) * n), 256, 0, s>>>(in, in_ns, out, out_ns, c, n, h, w);
  return cudaGetLastError();
}

cudaError_t dn_pool2_bwd(const float* dout, int64_t dout_ns, float* din, int64_t din_ns, int c, int n, int h,
                         int w, bool accumulate, cudaStream_t s) {
  k_pool2_bwd<<<blocks_for((int64_t)c * (h / 2) * (w / 2) * n), 256, 0, s>>>(dout, dout_ns, din, din_ns, c, n,
                                                                            h, w, accumulate ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t dn_up2(const float* in, int64_t in_ns, float* out, int64_t out_ns, int c, int n, int h, int w,
                   cudaStream_t s) {
  k_up2<<<blocks_for((int64_t)c * h * w * n), 256, 0, s>>>(in, in_ns, out, out_ns, c, n, h, w);
  return cudaGetLastError();
}

cudaError_t dn_up2_bwd(const float* dout, int64_t dout_ns, float* din, int64_t din_ns, int c, int n, int h,
                       int w, cudaStream_t s) {
  k_up2_bwd<<<blocks_for((int64_t)c * h * w * n), 256, 0, s>>>(dout, dout_ns, din, din_ns, c, n, h, w);
  return cudaGetLastError();
}

cudaError_t dn_mse(const float* pred, const float* target, int64_t count, float* grad, float* loss_sum,
                   cudaStream_t s) {
  const unsigned b = (unsigned)std::min<int64_t>(blocks_for(count), 148 * 8);
  k_mse<<<b, 256, 0, s>>>(pred, target, count, grad, loss_sum);
  return cudaGetLastError();
}

cudaError_t dn_adam(float* p, const float* g, float* m, float* v, int64_t count, float lr, float b1, float b2,
                    float eps, int step, cudaStream_t s) {
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  k_adam<<<blocks_for(count), 256, 0, s>>>(p, g, m, v, count, lr, b1, b2, eps, c1, c2);
  return cudaGetLastError();
}

}  // namespace pyr3
