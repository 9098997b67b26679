// Density estimation and tonemap passes (nvcc, sm_100a).
//
// Density estimation restates density_main (src/shaders/density.wgsl:51-123)
// in its scatter form: every non-empty bucket spreads
//   w(d) = exp(-d^2 / (2 sigma^2)) / knorm[r] * ls,   sigma = r / 3,
//   r = round(clamp(max_rad / (hits + 1)^curve, min_rad, max_rad)),
//   ls = k1 * log(1 + count * k2) / count
// over its own disc d^2 <= r^2.  The reference gathers (2R+1)^2 neighbours
// per output pixel; the scatter form does work proportional to each
// bucket's own disc, which is 10-1000x less on dense attractors.  Each CTA
// owns a TILE x TILE output tile accumulated in shared memory (float
// atomics); it streams the buckets of the tile plus an R halo with 128-bit
// loads, and small discs are splatted by the thread that read them while
// large discs are queued and splatted cooperatively by a whole warp.
// For kernel radii up to 31 (k_density_tma) the tile and its halo arrive in
// shared memory by one TMA tensor copy, every bucket is converted once, and
// the discs are sorted into radius classes: discs of radius 0-3 are spread
// as one flat list of (disc, tap) items, so every lane of every warp adds
// one tap, and larger discs are spread a warp at a time.
//
// Tonemap restates the visualize fragment shader (src/shaders/
// visualize_u32.wgsl:147-248 and visualize_f32.wgsl:162-271): fw x fw
// spatial-filter collapse of the super-res source (per-tap log-density ls
// for the raw histogram), flam3 alpha / vibrancy / highlight-power
// composite, background blend, clamp, then the colour curves (5 x 256 LUT:
// luma, r, g, b, composite, in the shader's order) and the HSL adjustment.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>

#include "passes.h"

namespace pyr3 {

// ------------------------------------------------------------- density
constexpr int kTile = 32;
constexpr int kDeThreads = 256;
constexpr int kBigQueue = 512;    // large-disc queue entries per tile
constexpr int kBigRadius = 3;     // discs with r > this go to the warp queue
constexpr int kKwMaxR = 64;       // weight table covers r <= 64

__device__ __forceinline__ int kw_offset(int r) {  // sum_{q<r} (q^2 + 1)
  return (r * (r - 1) * (2 * r - 1)) / 6 + r;
}

// kw_table[offset(r) + d2] = exp(-d2 / (2 sigma^2)) / max(knorm[r], 1e-6),
// exactly the reference's per-tap expression (density.wgsl:107-113).
__global__ void k_kw_table(const float* __restrict__ knorm, float* __restrict__ tab) {
  const int r = blockIdx.x;
  const float rad = (float)r;
  const float sig = fmaxf(rad / 3.0f, 1e-6f);
  const float kn = fmaxf(knorm[r], 1e-6f);
  for (int d2 = threadIdx.x; d2 <= r * r; d2 += blockDim.x) {
    const float kw = expf(-(float)d2 / (2.0f * sig * sig));
    tab[kw_offset(r) + d2] = kw / kn;
  }
}

struct DeBucket {
  int sx, sy, r;
  float4 v;  // hist RGBA * ls
};

// Accumulators of a tile: four planes (R, G, B, A) of kTile x kTile floats,
// so lanes adding into consecutive pixels of a row hit consecutive banks.
constexpr int kPlane = kTile * kTile;

__device__ __forceinline__ void de_disc(const DeBucket& b, int tx0, int ty0, float* acc,
                                        const float* __restrict__ tab, const float* __restrict__ knorm,
                                        int lane, int step) {
  // footprint of the disc clipped to the tile
  const int x0 = max(b.sx - b.r, tx0), x1 = min(b.sx + b.r, tx0 + kTile - 1);
  const int y0 = max(b.sy - b.r, ty0), y1 = min(b.sy + b.r, ty0 + kTile - 1);
  if (x0 > x1 || y0 > y1) return;
  const int wdt = x1 - x0 + 1;
  const int n = wdt * (y1 - y0 + 1);
  const int r2 = b.r * b.r;
  const float* row = b.r <= kKwMaxR ? tab + kw_offset(b.r) : nullptr;
  const float rad = (float)b.r;
  const float sig = fmaxf(rad / 3.0f, 1e-6f);
  const float kn = b.r <= kKwMaxR ? 0.0f : fmaxf(knorm[min(b.r, 256)], 1e-6f);
  for (int k = lane; k < n; k += step) {
    const int x = x0 + k % wdt, y = y0 + k / wdt;
    const int dx = x - b.sx, dy = y - b.sy;
    const int d2 = dx * dx + dy * dy;
    if (d2 > r2) continue;
    const float w = row ? row[d2] : expf(-(float)d2 / (2.0f * sig * sig)) / kn;
    float* a = acc + (y - ty0) * kTile + (x - tx0);
    atomicAdd(a, b.v.x * w);
    atomicAdd(a + kPlane, b.v.y * w);
    atomicAdd(a + 2 * kPlane, b.v.z * w);
    atomicAdd(a + 3 * kPlane, b.v.w * w);
  }
}

__global__ void __launch_bounds__(kDeThreads)
k_density(const uint4* __restrict__ hist, float4* __restrict__ out, DeParams p,
          const float* __restrict__ knorm, const float* __restrict__ tab) {
  __shared__ float acc[4 * kPlane];
  __shared__ DeBucket big[kBigQueue];
  __shared__ int n_big;
  const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTile;
  for (int i = threadIdx.x; i < 4 * kPlane; i += kDeThreads) acc[i] = 0.0f;
  if (threadIdx.x == 0) n_big = 0;
  __syncthreads();

  const int R = p.R;
  const int hx0 = max(tx0 - R, 0), hx1 = min(tx0 + kTile - 1 + R, (int)p.width - 1);
  const int hy0 = max(ty0 - R, 0), hy1 = min(ty0 + kTile - 1 + R, (int)p.height - 1);
  const int hw = hx1 - hx0 + 1;
  const int nsrc = hw * (hy1 - hy0 + 1);
  for (int s = threadIdx.x; s < nsrc; s += kDeThreads) {
    const int sx = hx0 + s % hw, sy = hy0 + s / hw;
    const uint4 h = hist[(size_t)sy * p.width + sx];
    const float nc = (float)h.w;
    if (nc <= 0.0f) continue;
    const float hits = nc / 255.0f;
    const float rf = fminf(fmaxf(p.max_rad / powf(hits + 1.0f, p.curve), p.min_rad), p.max_rad);
    const int r = min(max((int)rintf(rf), 0), 256);
    // disc misses the tile entirely
    if (sx + r < tx0 || sx - r > tx0 + kTile - 1 || sy + r < ty0 || sy - r > ty0 + kTile - 1) continue;
    const float ls = (p.k1 * logf(1.0f + nc * p.k2)) / nc;
    DeBucket b{sx, sy, r, make_float4((float)h.x * ls, (float)h.y * ls, (float)h.z * ls, nc * ls)};
    if (r > kBigRadius) {
      const int q = atomicAdd(&n_big, 1);
      if (q < kBigQueue) {
        big[q] = b;
        continue;
      }
    }
    de_disc(b, tx0, ty0, acc, tab, knorm, 0, 1);
  }
  __syncthreads();
  const int nb = min(n_big, kBigQueue);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int q = warp; q < nb; q += kDeThreads / 32) de_disc(big[q], tx0, ty0, acc, tab, knorm, lane, 32);
  __syncthreads();
  for (int i = threadIdx.x; i < kTile * kTile; i += kDeThreads) {
    const int x = tx0 + (i % kTile), y = ty0 + (i / kTile);
    if (x < (int)p.width && y < (int)p.height)
      out[(size_t)y * p.width + x] = make_float4(acc[i], acc[kPlane + i], acc[2 * kPlane + i], acc[3 * kPlane + i]);
  }
}

// ------------------------------------------------------------ TMA staging
// Tensor maps over an image of 16-byte RGBA buckets (u32 histogram or f32
// filtered sums) as a 3-D tensor: dim 0 the four 32-bit channels, dim 1 x,
// dim 2 y.  A box always starts at channel 0, so the innermost coordinate
// is 0 and 16-byte aligned; x and y may lie outside the image (a load
// fills zeros there).  No multicast: each CTA loads its own box.
__device__ __forceinline__ uint32_t sh_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tma_bar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n"
               "fence.mbarrier_init.release.cluster;\n" ::"r"(sh_addr(bar)) : "memory");
}

// One thread: announce `bytes` on the barrier and start the box copy at
// bucket (x, y) into dst (128-byte aligned shared memory).
__device__ __forceinline__ void tma_load_box(void* dst, const CUtensorMap* tm, int x, int y, uint64_t* bar,
                                             uint32_t bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n"
               ::"r"(sh_addr(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
               " [%0], [%1, {%2, %3, %4}], [%5];\n"
               ::"r"(sh_addr(dst)), "l"(reinterpret_cast<uint64_t>(tm)), "r"(0), "r"(x), "r"(y),
                 "r"(sh_addr(bar)) : "memory");
}

// Wait for phase 0 of the barrier; false once kTmaWaitLimit polls pass
// (a copy that never lands is reported, not waited for forever).
constexpr uint32_t kTmaWaitLimit = 1u << 24;
__device__ __forceinline__ bool tma_wait(uint64_t* bar) {
  for (uint32_t it = 0; it < kTmaWaitLimit; ++it) {
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n" : "=r"(done) : "r"(sh_addr(bar)) : "memory");
    if (done) return true;
  }
  return false;
}

// ------------------------------------------------ density, TMA-staged tile
constexpr int kDe2Classes = 5;   // discs of radius 0, 1, 2, 3, and >= 4
constexpr int kDe2Taps = 48;     // taps of the radius-0..3 discs: 1 + 5 + 13 + 29
constexpr uint16_t kDe2Skip = 0xffffu;
constexpr int kDe2MaxThreads = 1024;

size_t density_tma_smem(int R) {
  const size_t side = (size_t)kTile + 2 * (size_t)R, n = side * side;
  return n * 16 + (size_t)kTile * kTile * 16 + n * 4;
}

// Shared memory: the (32 + 2R)^2 halo (uint4 buckets, converted in place to
// the ls-scaled float4 each disc spreads), the 32 x 32 accumulator planes, the
// radius of each halo bucket (kDe2Skip: empty, or its disc misses the
// tile) and the halo indices sorted by radius class.
__global__ void __launch_bounds__(kDe2MaxThreads, 1)
k_density_tma(const __grid_constant__ CUtensorMap tm, float4* __restrict__ out, DeParams p,
              const float* __restrict__ knorm, const float* __restrict__ tab,
              unsigned long long* __restrict__ fault) {
  extern __shared__ __align__(128) unsigned char de_smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int cls_n[kDe2Classes], cls_off[kDe2Classes + 1], cls_cur[kDe2Classes];
  __shared__ signed char tap_dx[kDe2Taps], tap_dy[kDe2Taps];
  __shared__ unsigned char tap_d2[kDe2Taps];
  const int R = p.R, side = kTile + 2 * R, nsrc = side * side;
  float4* hv = (float4*)de_smem;
  float* acc = (float*)(hv + nsrc);
  uint16_t* rad = (uint16_t*)(acc + 4 * kPlane);
  uint16_t* idx = rad + nsrc;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5, nthr = (int)blockDim.x;
  const int tx0 = blockIdx.x * kTile, ty0 = blockIdx.y * kTile;
  const int hx0 = tx0 - R, hy0 = ty0 - R;

  if (t == 0) tma_bar_init(&bar);
  if (t < kDe2Classes) cls_n[t] = 0;
  if (t == 32) {  // taps of the discs of radius 0..3, row by row
    int n = 0;
    for (int r = 0; r <= 3; ++r)
      for (int dy = -r; dy <= r; ++dy)
        for (int dx = -r; dx <= r; ++dx)
          if (dx * dx + dy * dy <= r * r) {
            tap_dx[n] = (signed char)dx;
            tap_dy[n] = (signed char)dy;
            tap_d2[n] = (unsigned char)(dx * dx + dy * dy);
            ++n;
          }
  }
  for (int i = t; i < 4 * kPlane; i += nthr) acc[i] = 0.0f;
  __syncthreads();
  if (t == 0) tma_load_box(hv, &tm, hx0, hy0, &bar, (uint32_t)nsrc * 16u);
  if (!__syncthreads_and(tma_wait(&bar))) {
    // The copy did not land in time (the whole block agrees): report it,
    // wait once more (bounded) so no copy still writes this block's shared
    // memory, and mark the tile NaN rather than leave it stale.
    if (t == 0 && fault) atomicOr(fault, 8ull);
    tma_wait(&bar);
    const float nan = __int_as_float(0x7fc00000);
    for (int i = t; i < kTile * kTile; i += nthr) {
      const int x = tx0 + (i % kTile), y = ty0 + (i / kTile);
      if (x < (int)p.width && y < (int)p.height) out[(size_t)y * p.width + x] = make_float4(nan, nan, nan, nan);
    }
    return;
  }

  // Pass 1: radius, disc test and ls scaling of every halo bucket, in
  // place; class counts by warp ballots.
  for (int e0 = warp * 32; e0 < nsrc; e0 += nthr) {
    const int e = e0 + lane;
    int cls = -1;
    if (e < nsrc) {
      uint16_t rr = kDe2Skip;
      const float4 hb = hv[e];  // the raw bucket's bits (read and rewritten as float4)
      const uint4 h = make_uint4(__float_as_uint(hb.x), __float_as_uint(hb.y), __float_as_uint(hb.z),
                                 __float_as_uint(hb.w));
      const float nc = (float)h.w;
      if (nc > 0.0f) {
        const int sx = hx0 + e % side, sy = hy0 + e / side;
        const float hits = nc / 255.0f;
        const float rf = fminf(fmaxf(p.max_rad / powf(hits + 1.0f, p.curve), p.min_rad), p.max_rad);
        const int r = min(max((int)rintf(rf), 0), 256);
        if (!(sx + r < tx0 || sx - r > tx0 + kTile - 1 || sy + r < ty0 || sy - r > ty0 + kTile - 1)) {
          const float ls = (p.k1 * logf(1.0f + nc * p.k2)) / nc;
          hv[e] = make_float4((float)h.x * ls, (float)h.y * ls, (float)h.z * ls, nc * ls);
          rr = (uint16_t)r;
          cls = min(r, kDe2Classes - 1);
        }
      }
      rad[e] = rr;
    }
#pragma unroll
    for (int c = 0; c < kDe2Classes; ++c) {
      const unsigned m = __ballot_sync(0xffffffffu, cls == c);
      if (m && lane == __ffs(m) - 1) atomicAdd(&cls_n[c], __popc(m));
    }
  }
  __syncthreads();
  if (t == 0) {
    cls_off[0] = 0;
    for (int c = 0; c < kDe2Classes; ++c) {
      cls_off[c + 1] = cls_off[c] + cls_n[c];
      cls_cur[c] = cls_off[c];
    }
  }
  __syncthreads();
  // Pass 2: halo indices into class order.
  for (int e0 = warp * 32; e0 < nsrc; e0 += nthr) {
    const int e = e0 + lane;
    int cls = -1;
    if (e < nsrc && rad[e] != kDe2Skip) cls = min((int)rad[e], kDe2Classes - 1);
#pragma unroll
    for (int c = 0; c < kDe2Classes; ++c) {
      const unsigned m = __ballot_sync(0xffffffffu, cls == c);
      if (!m) continue;
      const int leader = __ffs(m) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(&cls_cur[c], __popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (cls == c) idx[base + __popc(m & ((1u << lane) - 1u))] = (uint16_t)e;
    }
  }
  __syncthreads();
  // Discs of radius 0..3: one item per (disc, tap), so all lanes work.
  const int n0 = cls_n[0], n1 = cls_n[1], n2 = cls_n[2], n3 = cls_n[3];
  const int e1 = n0, e2 = e1 + 5 * n1, e3 = e2 + 13 * n2, total = e3 + 29 * n3;
  for (int it = t; it < total; it += nthr) {
    int c, local, ntap, tap0;
    if (it < e1) { c = 0; local = it; ntap = 1; tap0 = 0; }
    else if (it < e2) { c = 1; local = it - e1; ntap = 5; tap0 = 1; }
    else if (it < e3) { c = 2; local = it - e2; ntap = 13; tap0 = 6; }
    else { c = 3; local = it - e3; ntap = 29; tap0 = 19; }
    const int disc = local / ntap, j = tap0 + (local - disc * ntap);
    const int e = idx[cls_off[c] + disc];
    const int x = hx0 + e % side + tap_dx[j], y = hy0 + e / side + tap_dy[j];
    if (x < tx0 || x >= tx0 + kTile || y < ty0 || y >= ty0 + kTile) continue;
    const float w = tab[kw_offset(c) + tap_d2[j]];
    const float4 v = hv[e];
    float* a = acc + (y - ty0) * kTile + (x - tx0);
    atomicAdd(a, v.x * w);
    atomicAdd(a + kPlane, v.y * w);
    atomicAdd(a + 2 * kPlane, v.z * w);
    atomicAdd(a + 3 * kPlane, v.w * w);
  }
  // Discs of radius >= 4: a warp each.
  for (int q = warp; q < cls_n[4]; q += nthr / 32) {
    const int e = idx[cls_off[4] + q];
    const DeBucket b{hx0 + e % side, hy0 + e / side, (int)rad[e], hv[e]};
    de_disc(b, tx0, ty0, acc, tab, knorm, lane, 32);
  }
  __syncthreads();
  for (int i = t; i < kPlane; i += nthr) {
    const int x = tx0 + (i % kTile), y = ty0 + (i / kTile);
    if (x < (int)p.width && y < (int)p.height)
      out[(size_t)y * p.width + x] = make_float4(acc[i], acc[kPlane + i], acc[2 * kPlane + i], acc[3 * kPlane + i]);
  }
}

// -------------------------------------------------------------- tonemap
__device__ __forceinline__ void rgb2hsv(const float c[3], float o[3]) {
  const float mx = fmaxf(fmaxf(c[0], c[1]), c[2]);
  const float mn = fminf(fminf(c[0], c[1]), c[2]);
  const float d = mx - mn;
  float h = 0.0f;
  if (d > 0.0f) {
    if (mx == c[0]) h = (c[1] - c[2]) / d;
    else if (mx == c[1]) h = 2.0f + (c[2] - c[0]) / d;
    else h = 4.0f + (c[0] - c[1]) / d;
    h *= 60.0f;
    if (h < 0.0f) h += 360.0f;
  }
  o[0] = h;
  o[1] = mx > 0.0f ? d / mx : 0.0f;
  o[2] = mx;
}

__device__ __forceinline__ void hsv2rgb(const float c[3], float o[3]) {
  const float h = c[0] / 60.0f, s = c[1], v = c[2];
  const float i = floorf(h), f = h - i;
  const float pp = v * (1.0f - s), q = v * (1.0f - s * f), t = v * (1.0f - s * (1.0f - f));
  float fi = i;  // WGSL i32(i) % 6 with a clamping conversion
  int ix = fi != fi ? 0 : (fi <= -2147483648.0f ? INT32_MIN : (fi >= 2147483520.0f ? 2147483520 : (int)fi));
  ix = ix % 6;
  switch (ix) {
    case 0: o[0] = v; o[1] = t; o[2] = pp; break;
    case 1: o[0] = q; o[1] = v; o[2] = pp; break;
    case 2: o[0] = pp; o[1] = v; o[2] = t; break;
    case 3: o[0] = pp; o[1] = q; o[2] = v; break;
    case 4: o[0] = t; o[1] = pp; o[2] = v; break;
    default: o[0] = v; o[1] = pp; o[2] = q; break;
  }
}

__device__ __forceinline__ float calc_alpha(float density, float g_inv, float linrange) {
  if (density <= 0.0f) return 0.0f;
  if (density < linrange) {
    const float funcval = powf(linrange, g_inv);
    const float frac = density / linrange;
    return (1.0f - frac) * density * (funcval / linrange) + frac * powf(density, g_inv);
  }
  return powf(density, g_inv);
}

__device__ __forceinline__ void calc_newrgb(const float c[3], float ls, float highpow, float o[3]) {
  if (ls == 0.0f || (c[0] == 0.0f && c[1] == 0.0f && c[2] == 0.0f)) {
    o[0] = o[1] = o[2] = 0.0f;
    return;
  }
  float sc[3];
  for (int i = 0; i < 3; ++i) sc[i] = ls * (c[i] / 255.0f);
  float maxa = sc[0], maxc = c[0] / 255.0f;
  if (sc[1] > maxa) { maxa = sc[1]; maxc = c[1] / 255.0f; }
  if (sc[2] > maxa) { maxa = sc[2]; maxc = c[2] / 255.0f; }
  if (maxa > 255.0f && highpow >= 0.0f) {
    const float newls = 255.0f / maxc;
    const float lsratio = powf(newls / ls, highpow);
    float nrgb[3], hsv[3];
    for (int i = 0; i < 3; ++i) nrgb[i] = newls * (c[i] / 255.0f) / 255.0f;
    rgb2hsv(nrgb, hsv);
    hsv[1] *= lsratio;
    hsv2rgb(hsv, nrgb);
    for (int i = 0; i < 3; ++i) o[i] = nrgb[i] * 255.0f;
  } else {
    const float newls = 255.0f / maxc;
    float adjhlp = -highpow;
    if (adjhlp > 1.0f) adjhlp = 1.0f;
    if (maxa <= 255.0f) adjhlp = 1.0f;
    const float k = (1.0f - adjhlp) * newls + adjhlp * ls;
    for (int i = 0; i < 3; ++i) o[i] = k * (c[i] / 255.0f);
  }
}

// Colour-curves lookup (visualize_u32.wgsl:51-56): linear between the two
// nearest of 256 entries of channel ch.
__device__ __forceinline__ float curve_lut(const float* __restrict__ lut, int ch, float x) {
  const float idx = fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f;
  const unsigned i0 = (unsigned)floorf(idx);
  const unsigned i1 = min(i0 + 1u, 255u);
  const float t = idx - (float)i0;
  return lut[ch * 256 + i0] * (1.0f - t) + lut[ch * 256 + i1] * t;
}

// ------------------------------------------------------- output kinds
// The display texture the reference renders to is rgba8unorm or
// rgba16float; its png16 and EXR exports transform the rgba16float readback
// on the host (src/gpu-readback.ts:83-115).  Here every kind is written by
// the pass that produces the fragment value.
__device__ __forceinline__ float to_half(float x) { return __half2float(__float2half_rn(x)); }

// displayHalfToPng16 (src/gpu-readback.ts:106-115) of one channel:
// round(clamp(h, 0, 1) * 65535), NaN -> 0.  Every binary16 in [0, 1] is
// k * 2^-24 with integer k, so the rounding is exact integer arithmetic:
// floor(k * 65535 / 2^24 + 1/2).
__device__ __forceinline__ uint16_t png16_sample(float x) {
  const float h = to_half(x);
  if (h != h) return 0;
  const uint64_t k = (uint64_t)(fminf(fmaxf(h, 0.0f), 1.0f) * 16777216.0f);
  return (uint16_t)((k * 65535ull + (1ull << 23)) >> 24);
}

// The clamp of displayHalfToLinearExr (src/gpu-readback.ts:90-93):
// non-finite -> 0, else clamp to [0, 1]; -0 becomes +0, as JS Math.max(0, -0)
// does (the + 0.0f).
__device__ __forceinline__ float exr_clamp(float x) {
  const float h = to_half(x);
  return fabsf(h) <= 65504.0f ? fminf(fmaxf(h, 0.0f), 1.0f) + 0.0f : 0.0f;
}

// srgbToLinear (src/srgb.ts:13-16) in double, as the reference computes
// it, rounded to f32 (its Float32Array).
__device__ __forceinline__ float srgb_to_linear(float c) {
  const double d = (double)c;
  return (float)(d <= 0.04045 ? d / 12.92 : pow((d + 0.055) / 1.055, 2.4));
}

template <int kOut>
__device__ __forceinline__ void store_pixel(const float o[4], void* __restrict__ out, size_t oi) {
  if (kOut == kOutRgba8) {
    uchar4 v;
    v.x = (unsigned char)__float2int_rn(o[0] * 255.0f);
    v.y = (unsigned char)__float2int_rn(o[1] * 255.0f);
    v.z = (unsigned char)__float2int_rn(o[2] * 255.0f);
    v.w = (unsigned char)__float2int_rn(o[3] * 255.0f);
    ((uchar4*)out)[oi] = v;
  } else if (kOut == kOutRgba32f) {
    ((float4*)out)[oi] = make_float4(o[0], o[1], o[2], o[3]);
  } else if (kOut == kOutRgba16f) {
    ushort4 v;
    v.x = __half_as_ushort(__float2half_rn(o[0]));
    v.y = __half_as_ushort(__float2half_rn(o[1]));
    v.z = __half_as_ushort(__float2half_rn(o[2]));
    v.w = __half_as_ushort(__float2half_rn(o[3]));
    ((ushort4*)out)[oi] = v;
  } else if (kOut == kOutPng16) {
    ((ushort4*)out)[oi] = make_ushort4(png16_sample(o[0]), png16_sample(o[1]), png16_sample(o[2]),
                                       png16_sample(o[3]));
  } else {  // kOutExrDisplay
    ((float4*)out)[oi] = make_float4(srgb_to_linear(exr_clamp(o[0])), srgb_to_linear(exr_clamp(o[1])),
                                     srgb_to_linear(exr_clamp(o[2])), exr_clamp(o[3]));
  }
}

// The fragment tail of visualize (visualize_u32.wgsl:160-248): alpha,
// vibrancy and highlight power from the filtered sums s0..s3, background,
// colour curves, HSL; stored at pixel oi as output kind kOut.
template <int kOut>
__device__ __forceinline__ void tonemap_pixel(float s0, float s1, float s2, float s3,
                                              const TonemapParams& p, const float* __restrict__ curves,
                                              void* __restrict__ out, size_t oi) {
  float o[4];
  if (s3 <= 0.0f) {
    if (p.transparent) { o[0] = o[1] = o[2] = o[3] = 0.0f; }
    else { o[0] = p.bg[0]; o[1] = p.bg[1]; o[2] = p.bg[2]; o[3] = 1.0f; }
  } else {
    const float g_inv = 1.0f / p.gamma;
    const float tmp = s3 / 255.0f;
    float alpha = calc_alpha(tmp, g_inv, p.linrange);
    const float ls_a = p.vibrancy * 256.0f * alpha / fmaxf(tmp, 1e-12f);
    alpha = fminf(fmaxf(alpha, 0.0f), 1.0f);
    const float c[3] = {s0, s1, s2};
    float nrgb[3];
    calc_newrgb(c, ls_a, p.highpow, nrgb);
    // At vibrancy 1 the per-channel gamma term is multiplied by
    // (1 - 1) * 256 = +0; with 0 < 1/gamma <= 1 its powf is finite for every
    // finite sum, so the product is +0 and is not computed.
    const bool no_perch = p.vibrancy == 1.0f && g_inv > 0.0f && g_inv <= 1.0f;
    for (int i = 0; i < 3; ++i) {
      const float perch =
          no_perch ? 0.0f : (1.0f - p.vibrancy) * 256.0f * powf(fmaxf(c[i] / 255.0f, 0.0f), g_inv);
      const float bg = p.transparent ? 0.0f : (1.0f - alpha) * 256.0f * p.bg[i];
      o[i] = fminf(fmaxf((nrgb[i] + perch + bg) / 256.0f, 0.0f), 1.0f);
    }
    if (p.curves_active) {  // visualize_u32.wgsl:217-231
      if (p.curves_active & 16u) {
        const float l = o[0] * 0.299f + o[1] * 0.587f + o[2] * 0.114f;
        const float ln = curve_lut(curves, 4, l);
        if (l > 0.0f) {
          const float k = ln / l;
          o[0] *= k; o[1] *= k; o[2] *= k;
        }
      }
      if (p.curves_active & 2u) o[0] = curve_lut(curves, 1, o[0]);
      if (p.curves_active & 4u) o[1] = curve_lut(curves, 2, o[1]);
      if (p.curves_active & 8u) o[2] = curve_lut(curves, 3, o[2]);
      if (p.curves_active & 1u) {
        o[0] = curve_lut(curves, 0, o[0]);
        o[1] = curve_lut(curves, 0, o[1]);
        o[2] = curve_lut(curves, 0, o[2]);
      }
    }
    if (p.hsl_active) {  // visualize_u32.wgsl:234-243
      float hsv[3];
      rgb2hsv(o, hsv);
      hsv[0] = hsv[0] + p.hsl_hue;
      hsv[0] = hsv[0] - 360.0f * floorf(hsv[0] / 360.0f);
      hsv[1] = fminf(fmaxf(hsv[1] * p.hsl_sat, 0.0f), 1.0f);
      hsv[2] = fminf(fmaxf(hsv[2] + p.hsl_light, 0.0f), 1.0f);
      hsv2rgb(hsv, o);
    }
    for (int i = 0; i < 3; ++i) o[i] = fminf(fmaxf(o[i], 0.0f), 1.0f);
    o[3] = p.transparent ? alpha : 1.0f;
  }
  store_pixel<kOut>(o, out, oi);
}

template <bool kU32, int kOut>
__global__ void __launch_bounds__(256)
k_tonemap(const uint4* __restrict__ hu, const float4* __restrict__ hf, TonemapParams p,
          const float* __restrict__ kern, const float* __restrict__ curves, void* __restrict__ out) {
  __shared__ float kk[kMaxTaps];
  if (threadIdx.x < p.fwidth) kk[threadIdx.x] = kern[threadIdx.x];
  __syncthreads();
  const uint32_t xi = blockIdx.x * 16 + (threadIdx.x & 15);
  const uint32_t yi = blockIdx.y * 16 + (threadIdx.x >> 4);
  if (xi >= p.width || yi >= p.height) return;
  const int N = (int)p.oversample, fw = (int)p.fwidth, half = fw / 2;
  const int sw = (int)p.width * N, sh = (int)p.height * N;
  const int cx = (int)xi * N + N / 2, cy = (int)yi * N + N / 2;
  float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
  for (int dy = 0; dy < fw; ++dy) {
    const float ky = kk[dy];
    const int sy = min(max(cy + dy - half, 0), sh - 1);
    for (int dx = 0; dx < fw; ++dx) {
      const float kx = kk[dx];
      const int sx = min(max(cx + dx - half, 0), sw - 1);
      const size_t sb = (size_t)sy * sw + sx;
      const float w = kx * ky;
      if (kU32) {
        const uint4 h = hu[sb];
        const float cnt = (float)h.w;
        if (cnt > 0.0f) {
          const float ls = (p.k1 * logf(1.0f + cnt * p.k2)) / cnt;
          s0 = s0 + ((float)h.x * ls) * w;
          s1 = s1 + ((float)h.y * ls) * w;
          s2 = s2 + ((float)h.z * ls) * w;
          s3 = s3 + (cnt * ls) * w;
        }
      } else {
        const float4 h = hf[sb];
        s0 = s0 + h.x * w;
        s1 = s1 + h.y * w;
        s2 = s2 + h.z * w;
        s3 = s3 + h.w * w;
      }
    }
  }
  tonemap_pixel<kOut>(s0, s1, s2, s3, p, curves, out, (size_t)yi * p.width + xi);
}

// The same pass with the block's super-sampled tile staged in shared
// memory: a block of T x T output pixels first reads the (T-1)N + fw square
// of source buckets its filter taps cover (edge-clamped, coalesced rows),
// converting each raw bucket to its log-density-scaled RGBA once, then
// every pixel gathers its fw x fw taps from shared memory.  The taps are
// added in the same order with the same products as k_tonemap, so the
// output is the same bit for bit; each bucket is read from HBM once per
// block instead of once per tap (about (fw/N)^2 times), and its logf is
// taken once instead of per tap.
template <bool kU32, int kOut>
__global__ void __launch_bounds__(256)
k_tonemap_tile(const uint4* __restrict__ hu, const float4* __restrict__ hf, TonemapParams p,
               const float* __restrict__ kern, const float* __restrict__ curves, void* __restrict__ out,
               int T, int side, const __grid_constant__ CUtensorMap tm, int use_tma,
               unsigned long long* __restrict__ fault) {
  extern __shared__ __align__(128) float4 tile[];  // side x side
  __shared__ float kk[kMaxTaps];
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x < p.fwidth) kk[threadIdx.x] = kern[threadIdx.x];
  const int N = (int)p.oversample, fw = (int)p.fwidth, half = fw / 2;
  const int sw = (int)p.width * N, sh = (int)p.height * N;
  const int ox = (int)blockIdx.x * T * N + N / 2 - half, oy = (int)blockIdx.y * T * N + N / 2 - half;
  const int n = side * side, nt = (int)blockDim.x;
  // A tile whose source square lies inside the image arrives by one TMA
  // tensor copy (then converted in place); an edge tile, whose taps clamp to
  // the border, reads its square with clamped loads.
  if (use_tma && ox >= 0 && oy >= 0 && ox + side <= sw && oy + side <= sh) {
    if (threadIdx.x == 0) tma_bar_init(&bar);
    __syncthreads();
    if (threadIdx.x == 0) tma_load_box(tile, &tm, ox, oy, &bar, (uint32_t)n * 16u);
    if (!__syncthreads_and(tma_wait(&bar))) {
      if (threadIdx.x == 0 && fault) atomicOr(fault, 16ull);
      tma_wait(&bar);
      const float nan = __int_as_float(0x7fc00000);
      const float o[4] = {nan, nan, nan, nan};
      const uint32_t xi = blockIdx.x * T + (int)threadIdx.x % T, yi = blockIdx.y * T + (int)threadIdx.x / T;
      if (xi < p.width && yi < p.height) store_pixel<kOut>(o, out, (size_t)yi * p.width + xi);
      return;
    }
    if (kU32) {
      for (int e = threadIdx.x; e < n; e += nt) {
        const float4 b = tile[e];
        const float cnt = (float)__float_as_uint(b.w);
        float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (cnt > 0.0f) {
          const float ls = (p.k1 * logf(1.0f + cnt * p.k2)) / cnt;
          v = make_float4((float)__float_as_uint(b.x) * ls, (float)__float_as_uint(b.y) * ls,
                          (float)__float_as_uint(b.z) * ls, cnt * ls);
        }
        tile[e] = v;
      }
    }
  } else
  // Four loads in flight per thread, then the conversions.
  for (int e0 = threadIdx.x; e0 < n; e0 += 4 * nt) {
    uint4 raw[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int e = e0 + j * nt;
      if (e < n) {
        const int ty = e / side, tx = e - ty * side;
        const int sy = min(max(oy + ty, 0), sh - 1), sx = min(max(ox + tx, 0), sw - 1);
        const size_t sb = (size_t)sy * sw + sx;
        raw[j] = kU32 ? hu[sb] : reinterpret_cast<const uint4*>(hf)[sb];
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int e = e0 + j * nt;
      if (e >= n) break;
      float4 v;
      if (kU32) {
        const uint4 h = raw[j];
        const float cnt = (float)h.w;
        if (cnt > 0.0f) {
          const float ls = (p.k1 * logf(1.0f + cnt * p.k2)) / cnt;
          v = make_float4((float)h.x * ls, (float)h.y * ls, (float)h.z * ls, cnt * ls);
        } else {
          v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // adds +0 to sums that are >= +0
        }
      } else {
        v = make_float4(__uint_as_float(raw[j].x), __uint_as_float(raw[j].y), __uint_as_float(raw[j].z),
                        __uint_as_float(raw[j].w));
      }
      tile[e] = v;
    }
  }
  __syncthreads();
  const int lx = (int)threadIdx.x % T, ly = (int)threadIdx.x / T;
  const uint32_t xi = blockIdx.x * T + lx, yi = blockIdx.y * T + ly;
  if (xi >= p.width || yi >= p.height) return;
  float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
  for (int dy = 0; dy < fw; ++dy) {
    const float ky = kk[dy];
    const float4* row = tile + (ly * N + dy) * side + lx * N;
    for (int dx = 0; dx < fw; ++dx) {
      const float kx = kk[dx];
      const float w = kx * ky;
      const float4 v = row[dx];
      s0 = s0 + v.x * w;
      s1 = s1 + v.y * w;
      s2 = s2 + v.z * w;
      s3 = s3 + v.w * w;
    }
  }
  tonemap_pixel<kOut>(s0, s1, s2, s3, p, curves, out, (size_t)yi * p.width + xi);
}

// -------------------------------------------------------------- launch
cudaError_t build_kw_table(const float* knorm, float* tab, cudaStream_t s) {
  k_kw_table<<<kKwMaxR + 1, 256, 0, s>>>(knorm, tab);
  return cudaGetLastError();
}

size_t kw_table_floats() { return (size_t)(kKwMaxR * (kKwMaxR + 1) * (2 * kKwMaxR + 1)) / 6 + kKwMaxR + 1 + 1; }

namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                  CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links no driver library); null if the driver has none.
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return (EncodeTiledFn)f;
  }();
  return fn;
}
}  // namespace

bool encode_bucket_map(CUtensorMap* tm, const void* base, uint32_t width, uint32_t height, uint32_t box_w,
                       uint32_t box_h) {
  const EncodeTiledFn fn = encode_tiled();
  if (!fn || ((uintptr_t)base & 15u) || box_w < 1 || box_w > 256 || box_h < 1 || box_h > 256) return false;
  const cuuint64_t dims[3] = {4, width, height};
  const cuuint64_t strides[2] = {16, (cuuint64_t)width * 16};
  const cuuint32_t box[3] = {4, box_w, box_h};
  const cuuint32_t estride[3] = {1, 1, 1};
  return fn(tm, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, const_cast<void*>(base), dims, strides, box, estride,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_density(const uint32_t* hist, float* filtered, const DeParams& p,
                           const float* knorm, const float* tab, unsigned long long* fault, cudaStream_t s) {
  dim3 grid((p.width + kTile - 1) / kTile, (p.height + kTile - 1) / kTile);
  // The TMA-staged kernel where its tile fits in shared memory (kernel
  // radius up to kDensityTmaMaxR); the streaming kernel otherwise.
  if (p.R >= 0 && p.R <= kDensityTmaMaxR) {
    CUtensorMap tm;
    const uint32_t side = (uint32_t)(kTile + 2 * p.R);
    if (encode_bucket_map(&tm, hist, p.width, p.height, side, side)) {
      const size_t smem = density_tma_smem(p.R);
      static bool attr_set[64] = {};  // per device: the attribute belongs to the current device
      int dev = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e != cudaSuccess) return e;
      if (dev < 0 || dev >= 64 || !attr_set[dev]) {
        e = cudaFuncSetAttribute(k_density_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)density_tma_smem(kDensityTmaMaxR));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr_set[dev] = true;
      }
      // 512 threads where three blocks fit on an SM (48 warps), 1024 where
      // the halo leaves room for one block only (32 warps).
      const unsigned thr = smem <= 75 * 1024 ? 512u : 1024u;
      k_density_tma<<<grid, thr, smem, s>>>(tm, (float4*)filtered, p, knorm, tab, fault);
      return cudaGetLastError();
    }
  }
  k_density<<<grid, kDeThreads, 0, s>>>((const uint4*)hist, (float4*)filtered, p, knorm, tab);
  return cudaGetLastError();
}

namespace {
template <int kOut>
void tonemap_launch(const uint32_t* hist_u32, const float* filtered, const TonemapParams& p,
                    const float* kern, const float* curves, void* out, int T, int side,
                    unsigned long long* fault, cudaStream_t s) {
  if (T) {
    dim3 grid((p.width + T - 1) / T, (p.height + T - 1) / T);
    const size_t smem = (size_t)side * side * sizeof(float4);
    const unsigned thr = (unsigned)(T * T);
    CUtensorMap tm;
    const void* src = hist_u32 ? (const void*)hist_u32 : (const void*)filtered;
    const int use_tma = encode_bucket_map(&tm, src, p.width * p.oversample, p.height * p.oversample,
                                          (uint32_t)side, (uint32_t)side) ? 1 : 0;
    if (!use_tma) std::memset(&tm, 0, sizeof tm);
    if (hist_u32)
      k_tonemap_tile<true, kOut><<<grid, thr, smem, s>>>((const uint4*)hist_u32, nullptr, p, kern, curves, out, T,
                                                         side, tm, use_tma, fault);
    else
      k_tonemap_tile<false, kOut><<<grid, thr, smem, s>>>(nullptr, (const float4*)filtered, p, kern, curves, out,
                                                          T, side, tm, use_tma, fault);
    return;
  }
  dim3 grid((p.width + 15) / 16, (p.height + 15) / 16);
  if (hist_u32)
    k_tonemap<true, kOut><<<grid, 256, 0, s>>>((const uint4*)hist_u32, nullptr, p, kern, curves, out);
  else
    k_tonemap<false, kOut><<<grid, 256, 0, s>>>(nullptr, (const float4*)filtered, p, kern, curves, out);
}

template <int kOut>
__global__ void __launch_bounds__(256) k_convert_display(const float4* __restrict__ in, uint64_t n,
                                                         void* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (uint64_t)gridDim.x * 256) {
    const float4 v = in[i];
    const float o[4] = {v.x, v.y, v.z, v.w};
    store_pixel<kOut>(o, out, i);
  }
}
}  // namespace

size_t out_bytes_per_pixel(int out_kind) {
  switch (out_kind) {
    case kOutRgba8: return 4;
    case kOutRgba16f:
    case kOutPng16: return 8;
    case kOutRgba32f:
    case kOutExrDisplay: return 16;
    default: return 0;
  }
}

cudaError_t launch_tonemap(const uint32_t* hist_u32, const float* filtered, const TonemapParams& p,
                           const float* kern, const float* curves, void* out, int out_kind,
                           unsigned long long* fault, cudaStream_t s) {
  // Shared-memory tile of 16 x 16 (else 8 x 8) output pixels when its source
  // square fits in 48 KB; the per-tap gather otherwise (large oversample
  // with a wide filter).
  const int N = (int)p.oversample, fw = (int)p.fwidth;
  int T = 0, side = 0;
  for (int t : {16, 8}) {
    const int sd = (t - 1) * N + fw;
    if ((size_t)sd * sd * sizeof(float4) <= 48 * 1024) {
      T = t;
      side = sd;
      break;
    }
  }
  switch (out_kind) {
    case kOutRgba8: tonemap_launch<kOutRgba8>(hist_u32, filtered, p, kern, curves, out, T, side, fault, s); break;
    case kOutRgba32f: tonemap_launch<kOutRgba32f>(hist_u32, filtered, p, kern, curves, out, T, side, fault, s); break;
    case kOutRgba16f: tonemap_launch<kOutRgba16f>(hist_u32, filtered, p, kern, curves, out, T, side, fault, s); break;
    case kOutPng16: tonemap_launch<kOutPng16>(hist_u32, filtered, p, kern, curves, out, T, side, fault, s); break;
    case kOutExrDisplay: tonemap_launch<kOutExrDisplay>(hist_u32, filtered, p, kern, curves, out, T, side, fault, s); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_convert_display(const float* in, uint64_t pixels, int out_kind, void* out, int sms,
                                   cudaStream_t s) {
  if (pixels == 0) return cudaSuccess;
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((pixels + 255) / 256, (uint64_t)sms * 8));
  const float4* src = (const float4*)in;
  switch (out_kind) {
    case kOutRgba8: k_convert_display<kOutRgba8><<<grid, 256, 0, s>>>(src, pixels, out); break;
    case kOutRgba32f: k_convert_display<kOutRgba32f><<<grid, 256, 0, s>>>(src, pixels, out); break;
    case kOutRgba16f: k_convert_display<kOutRgba16f><<<grid, 256, 0, s>>>(src, pixels, out); break;
    case kOutPng16: k_convert_display<kOutPng16><<<grid, 256, 0, s>>>(src, pixels, out); break;
    case kOutExrDisplay: k_convert_display<kOutExrDisplay><<<grid, 256, 0, s>>>(src, pixels, out); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------- linear export
__global__ void __launch_bounds__(256)
k_linear_export(const uint4* __restrict__ hist, uint32_t width, uint32_t height, uint32_t os,
                double scale, float4* __restrict__ out) {
  const uint32_t x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 16 + (threadIdx.x >> 4);
  if (x >= width || y >= height) return;
  const size_t sw = (size_t)width * os;
  double r = 0.0, g = 0.0, b = 0.0, c = 0.0;  // integer sums: exact in f64
  for (uint32_t sy = 0; sy < os; ++sy)
    for (uint32_t sx = 0; sx < os; ++sx) {
      const uint4 h = hist[((size_t)y * os + sy) * sw + (size_t)x * os + sx];
      r += (double)h.x;
      g += (double)h.y;
      b += (double)h.z;
      c += (double)h.w;
    }
  const double a = c * scale;
  out[(size_t)y * width + x] = make_float4((float)(r * scale), (float)(g * scale), (float)(b * scale),
                                           (float)(a < 0.0 ? 0.0 : (a > 1.0 ? 1.0 : a)));
}

cudaError_t launch_linear_export(const uint32_t* hist, uint32_t width, uint32_t height,
                                 uint32_t oversample, double k1, double k2, float* out,
                                 cudaStream_t s) {
  const double scale = (k1 * k2) / (double)(oversample * oversample);
  dim3 grid((width + 15) / 16, (height + 15) / 16);
  k_linear_export<<<grid, 256, 0, s>>>((const uint4*)hist, width, height, oversample, scale,
                                       (float4*)out);
  return cudaGetLastError();
}


namespace {
// Each thread walks an LCG over cells and deposits 1 into the 4 channels of
// each, with the chaos kernel's saturation check on the returned values.
__global__ void __launch_bounds__(256) k_splat_rate(uint32_t* cells, uint64_t n_cells, uint64_t per_thread,
                                                    uint64_t extra) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t n = per_thread + (tid < extra ? 1 : 0);
  uint32_t x = (uint32_t)(tid * 2654435761ull) ^ 0x9e3779b9u;
  for (uint64_t i = 0; i < n; ++i) {
    x = x * 1664525u + 1013904223u;
    uint32_t* c = cells + ((uint64_t)x * n_cells >> 32) * 4;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t old = atomicAdd(c + k, 1u);
      if (old > 0xffffffffu - 1u) atomicOr(c + k, 0xffffffffu);
    }
  }
}
}  // namespace

cudaError_t launch_splat_rate(uint32_t* cells, uint64_t n_cells, uint64_t splats, int sms, cudaStream_t s) {
  const uint64_t threads = (uint64_t)sms * 8 * 256;
  k_splat_rate<<<(unsigned)(sms * 8), 256, 0, s>>>(cells, n_cells, splats / threads, splats % threads);
  return cudaGetLastError();
}

// ------------------------------------------------------------ luminance
namespace {
__device__ __forceinline__ uint32_t rgb8_sum(uint32_t px) {
  return (px & 0xffu) + ((px >> 8) & 0xffu) + ((px >> 16) & 0xffu);
}

// One channel of an rgba32f pixel as the reference reads it back from an
// rgba16float texture: rounded to binary16, non-finite -> 0, clamped to
// [0, 1]; in units of 2^-24.
__device__ __forceinline__ uint32_t half_units(float x) {
  const float h = __half2float(__float2half_rn(x));
  if (!(fabsf(h) <= 65504.0f)) return 0u;
  return (uint32_t)(fminf(fmaxf(h, 0.0f), 1.0f) * 16777216.0f);
}

__device__ __forceinline__ uint32_t half_bits_units(uint32_t bits) {
  return half_units(__half2float(__ushort_as_half((unsigned short)bits)));
}

// R + G + B of the pixels in one 16-byte word: 4 rgba8 pixels, 1 rgba32f
// pixel or 2 rgba16f pixels.
template <int kKind>
__device__ __forceinline__ uint64_t word_luma(const uint4 v) {
  if (kKind == kOutRgba8) return rgb8_sum(v.x) + rgb8_sum(v.y) + rgb8_sum(v.z) + rgb8_sum(v.w);
  if (kKind == kOutRgba32f)
    return (uint64_t)half_units(__uint_as_float(v.x)) + half_units(__uint_as_float(v.y)) +
           half_units(__uint_as_float(v.z));
  return (uint64_t)half_bits_units(v.x & 0xffffu) + half_bits_units(v.x >> 16) + half_bits_units(v.y & 0xffffu) +
         half_bits_units(v.z & 0xffffu) + half_bits_units(v.z >> 16) + half_bits_units(v.w & 0xffffu);
}

// Grid-stride over 16-byte words, four independent loads in flight per
// thread; the pixels after the last whole word (rgba8: up to 3 as u32,
// rgba16f: 1 as two u32) are added by block 0; one atomic per block.
template <int kKind>
__global__ void __launch_bounds__(256) k_luma_sum(const uint4* __restrict__ img, uint64_t words,
                                                  const uint32_t* __restrict__ tail, uint32_t n_tail,
                                                  unsigned long long* sum) {
  const uint64_t stride = (uint64_t)gridDim.x * 256;
  uint64_t acc = 0;
  uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
  for (; i + 3 * stride < words; i += 4 * stride) {
    const uint4 a = __ldcs(img + i), b = __ldcs(img + i + stride), c = __ldcs(img + i + 2 * stride),
                d = __ldcs(img + i + 3 * stride);
    acc += word_luma<kKind>(a) + word_luma<kKind>(b) + word_luma<kKind>(c) + word_luma<kKind>(d);
  }
  for (; i < words; i += stride) acc += word_luma<kKind>(__ldcs(img + i));
  if (blockIdx.x == 0 && threadIdx.x < n_tail) {
    if (kKind == kOutRgba8) acc += rgb8_sum(tail[threadIdx.x]);
    if (kKind == kOutRgba16f)
      acc += (uint64_t)half_bits_units(tail[0] & 0xffffu) + half_bits_units(tail[0] >> 16) +
             half_bits_units(tail[1] & 0xffffu);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  __shared__ uint64_t warp_sums[8];
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t t = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) t += warp_sums[w];
    atomicAdd(sum, (unsigned long long)t);
  }
}
}  // namespace

cudaError_t launch_luma_sum(const void* img, uint64_t pixels, int kind, unsigned long long* sum,
                            int sms, cudaStream_t s) {
  const uint64_t per_word = kind == kOutRgba8 ? 4 : kind == kOutRgba16f ? 2 : 1;
  const uint64_t words = pixels / per_word;
  const uint32_t n_tail = (uint32_t)(pixels - words * per_word);
  const uint64_t want = (words + 255) / 256;
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms * 8));
  const uint32_t* tail = (const uint32_t*)((const uint4*)img + words);
  switch (kind) {
    case kOutRgba8: k_luma_sum<kOutRgba8><<<grid, 256, 0, s>>>((const uint4*)img, words, tail, n_tail, sum); break;
    case kOutRgba32f: k_luma_sum<kOutRgba32f><<<grid, 256, 0, s>>>((const uint4*)img, words, nullptr, 0, sum); break;
    case kOutRgba16f: k_luma_sum<kOutRgba16f><<<grid, 256, 0, s>>>((const uint4*)img, words, tail, n_tail, sum); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
}  // namespace pyr3
