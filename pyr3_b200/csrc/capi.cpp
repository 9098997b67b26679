// pyr3-b200 C-ABI (include/pyr3.h): renderer lifecycle, the iterate /
// present path, and stage entry points for parity tests.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "jit.h"
#include "denoise.h"
#include "noalloc.h"
#include "passes.h"
#include "pyr3.h"

#define PYR3_API extern "C" __attribute__((visibility("default")))

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CUDA_TRY(expr)                                                            \
  do {                                                                            \
    cudaError_t e_ = (expr);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(e_ == cudaErrorMemoryAllocation ? PYR3_E_NOMEM : PYR3_E_CUDA,   \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));            \
  } while (0)

// Launch a kernel of a JIT-loaded library (cudaKernel_t).
#define LAUNCH_TRY(kernel, grid, block, smem, stream, args)                       \
  CUDA_TRY(cudaLaunchKernel((const void*)(kernel), dim3(grid), dim3(block), args, smem, stream))

constexpr uint32_t kGrain = 16384;
constexpr uint32_t kFuse = 200;         // src/renderer.ts:41
constexpr float kDefaultJitter = 1e-7f; // src/chaos.ts:96
constexpr int kWpb = 256;
// Launches of at least this many samples may run the kernel autotuner.
constexpr uint64_t kTuneMinSamples = 64ull << 20;

// Host mirror of the NVRTC kernel's argument block (layout must match
// ChaosArgs in csrc/jit/chaos_kernel.cuh).
struct ChaosArgs {
  uint32_t* hist;
  uint32_t* idx_sum;
  const float* palette;
  const unsigned short* pick_start;
  uint64_t walker_base, n_walkers, iters_base, iters_extra;
  uint32_t fuse;
  uint32_t width, height;
  float scale, cx, cy;
  float cos_r, sin_r;
  uint32_t seed;
  float jitter;
  uint32_t palette_mode;
  uint32_t capture_index;
  uint32_t color_mode;
  float flow_strength, flow_scale;
  uint32_t trap_kind, trap_mode;
  float trap_cx, trap_cy, trap_radius, trap_nx, trap_ny, trap_falloff, trap_freq, trap_strength;
  float phase_strength, phase_freq;
  float xform_blend;
  uint64_t* counters;
  uint64_t* sched;
  uint32_t* wrec;
  uint32_t cta_slots;
};

// Host mirror of WaveArgs in csrc/jit/chaos_kernel.cuh (the wave kernel's
// second argument block).
struct WaveArgs {
  uint32_t* st;
  uint32_t* cnt;
  uint64_t cap;
  uint32_t mode;
  uint32_t rd_buf, wr_buf;
  uint32_t rd_cnt, wr_cnt, zero_cnt;
};
static_assert(sizeof(WaveArgs) == 48, "WaveArgs layout");

// ---- host restatements of the reference's host-side math --------------
// Pick table (src/genome.ts:482-534) as per-row boundaries: start[r][j] is
// the first grain index whose table entry is >= j, so the device recovers
// the 16384-entry table exactly (see pick_xform in chaos_kernel.cuh).
bool build_pick_starts(int n, const float* weights_f, const float* xaos, std::vector<uint16_t>* out,
                       std::string* err) {
  std::vector<double> w(n);
  for (int i = 0; i < n; ++i) w[i] = (double)weights_f[i];
  out->assign((size_t)(n + 1) * n, (uint16_t)kGrain);
  std::vector<uint32_t> row(kGrain);
  for (int r = 0; r <= n; ++r) {
    const int xi = r < n ? r : -1;
    auto mult = [&](int j) -> double {
      return (xi >= 0 && xaos && j < n) ? (double)xaos[(size_t)xi * n + j] : 1.0;
    };
    double sum = 0.0;
    for (int i = 0; i < n; ++i) {
      double d = w[i] * mult(i);
      if (!std::isfinite(d) || d < 0) {
        *err = "xform weight must be non-negative finite";
        return false;
      }
      sum += d;
    }
    std::fill(row.begin(), row.end(), 0u);
    if (sum != 0.0) {
      const double dr = sum / kGrain;
      int j = 0;
      double t = w[0] * mult(0), acc = 0.0;
      for (uint32_t g = 0; g < kGrain; ++g) {
        while (acc >= t && j <= n) {
          ++j;
          t += (j < n ? w[j] : 0.0) * mult(j);
        }
        row[g] = (uint32_t)std::min(j, n - 1);
        acc += dr;
      }
    }
    uint16_t* st = out->data() + (size_t)r * n;
    st[0] = 0;
    for (int j = 1; j < n; ++j) {
      uint32_t g = 0;
      while (g < kGrain && row[g] < (uint32_t)j) ++g;
      st[j] = (uint16_t)g;
    }
  }
  return true;
}

// src/density.ts:78-99.
void kernel_norm_lut(float* out) {
  for (int r = 0; r <= 256; ++r) {
    if (r == 0) {
      out[0] = 1.0f;
      continue;
    }
    const double sigma = r / 3.0, inv2s2 = 1.0 / (2.0 * sigma * sigma), r2 = (double)r * r;
    double sum = 0.0;
    for (int dy = -r; dy <= r; ++dy)
      for (int dx = -r; dx <= r; ++dx) {
        const double d2 = (double)dx * dx + (double)dy * dy;
        if (d2 <= r2) sum += std::exp(-d2 * inv2s2);
      }
    out[r] = (float)sum;
  }
}

// src/spatial-filter.ts:217-256 (gaussian shape).
int spatial_kernel(double radius, int os, float* out) {
  const double supp = 1.5;
  const double fw = 2.0 * supp * os * radius;
  int fwidth = (int)std::floor(fw) + 1;
  if (((fwidth ^ os) & 1) != 0) fwidth++;
  fwidth = std::max(3, std::min(pyr3::kMaxTaps, fwidth));
  const double adjust = fw > 0 ? (supp * fwidth) / fw : 1.0;
  double v[pyr3::kMaxTaps], sum = 0.0;
  for (int i = 0; i < fwidth; ++i) {
    const double x = ((2.0 * i + 1.0) / fwidth - 1.0) * adjust;
    v[i] = std::exp(-2.0 * x * x);
    sum += v[i];
  }
  for (int i = 0; i < fwidth; ++i) {
    const float tap = (float)v[i];
    out[i] = sum != 0 ? (float)((double)tap / sum) : tap;
  }
  return fwidth;
}

int g_num_sms = 0;

int device_sms(int dev) {
  if (g_num_sms == 0) cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
  return g_num_sms > 0 ? g_num_sms : 148;
}

int g_l2_bytes = 0;

// L2 size in bytes (about 126.5 MiB on B200).
uint64_t device_l2(int dev) {
  if (g_l2_bytes == 0) cudaDeviceGetAttribute(&g_l2_bytes, cudaDevAttrL2CacheSize, dev);
  return g_l2_bytes > 0 ? (uint64_t)g_l2_bytes : (126ull << 20);
}

}  // namespace

struct pyr3_renderer {
  int device = 0;
  uint32_t W = 0, H = 0, os = 1, SW = 0, SH = 0;
  float filter_radius = 0.5f;
  int fwidth = 3;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  uint32_t* d_hist = nullptr;
  uint32_t* d_idx = nullptr;
  float* d_filtered = nullptr;
  float* d_pal = nullptr;
  float* d_knorm = nullptr;
  float* d_kwtab = nullptr;
  float* d_kern = nullptr;
  float* d_curves = nullptr;  // 5 x 256 colour-curves LUT
  void* d_out = nullptr;
  size_t out_bytes = 0;
  uint16_t* d_pick = nullptr;
  size_t pick_cap = 0;
  uint64_t* d_counters = nullptr;
  uint64_t* d_sched = nullptr;  // queue kernel: [0] walkers handed out, [1] sticky fault flags
  unsigned long long* d_luma = nullptr;  // luminance sum (auto-exposure)
  unsigned long long* h_luma = nullptr;  // its pinned host copy
  uint32_t* d_wrec = nullptr;   // queue kernel: walker records (CTAs x slots)
  uint32_t* d_wave = nullptr;   // wave kernel: per population walker state + region counts
  size_t wave_bytes = 0;
  cudaStream_t wave_aux = nullptr;  // wave kernel: the second population's stream
  cudaEvent_t wave_fork = nullptr, wave_join = nullptr;
  size_t wrec_cap = 0;
  bool capture = false;
  float last_ms = 0.0f;
  uint64_t last_launches = 0;  // kernel launches of the last pyr3_iterate
  cudaEvent_t marks[8] = {};
  cudaEvent_t tune[4] = {};  // kernel autotuner
  void* d_flush = nullptr;
  size_t flush_bytes = 0;
  std::vector<std::shared_ptr<pyr3::ChaosModule>> modules;  // keep-alive
};

namespace {

void free_buffers(pyr3_renderer* r) {
  cudaFree(r->d_hist);
  cudaFree(r->d_idx);
  cudaFree(r->d_filtered);
  cudaFree(r->d_out);
  r->d_hist = r->d_idx = nullptr;
  r->d_filtered = nullptr;
  r->d_out = nullptr;
  r->out_bytes = 0;
}

int alloc_buffers(pyr3_renderer* r, const pyr3_opts* o) {
  if (!o || o->width == 0 || o->height == 0 || o->oversample == 0)
    return fail(PYR3_E_INVALID, "width, height and oversample must be positive");
  if ((uint64_t)o->width * o->oversample > 65535 || (uint64_t)o->height * o->oversample > 65535)
    return fail(PYR3_E_INVALID, "super-res canvas exceeds 65535 pixels per side");
  r->W = o->width;
  r->H = o->height;
  r->os = o->oversample;
  r->SW = r->W * r->os;
  r->SH = r->H * r->os;
  r->filter_radius = o->filter_radius > 0 ? o->filter_radius : 0.5f;
  float kern[pyr3::kMaxTaps];
  r->fwidth = spatial_kernel(r->filter_radius, (int)r->os, kern);
  const size_t n = (size_t)r->SW * r->SH;
  CUDA_TRY(cudaMalloc(&r->d_hist, n * 16));
  CUDA_TRY(cudaMalloc(&r->d_idx, n * 4));
  CUDA_TRY(cudaMemsetAsync(r->d_hist, 0, n * 16, r->stream));
  CUDA_TRY(cudaMemsetAsync(r->d_idx, 0, n * 4, r->stream));
  CUDA_TRY(cudaMemcpyAsync(r->d_kern, kern, sizeof kern, cudaMemcpyHostToDevice, r->stream));
  return PYR3_OK;
}

int ensure_filtered(pyr3_renderer* r) {
  if (!r->d_filtered) CUDA_TRY(cudaMalloc(&r->d_filtered, (size_t)r->SW * r->SH * 16));
  return PYR3_OK;
}

int ensure_out(pyr3_renderer* r, size_t bytes) {
  if (r->out_bytes < bytes) {
    cudaFree(r->d_out);
    r->d_out = nullptr;
    CUDA_TRY(cudaMalloc(&r->d_out, bytes));
    r->out_bytes = bytes;
  }
  return PYR3_OK;
}

int set_device(int dev) {
  CUDA_TRY(cudaSetDevice(dev));
  CUDA_TRY(cudaFree(nullptr));  // create / bind the primary context for the driver API
  return PYR3_OK;
}

}  // namespace

// ---------------------------------------------------------------- lifecycle
PYR3_API const char* pyr3_last_error(void) { return g_err.c_str(); }

PYR3_API int pyr3_create(const pyr3_opts* opts, pyr3_renderer** out) {
  if (!opts || !out) return fail(PYR3_E_INVALID, "null argument");
  int rc = set_device(opts->device);
  if (rc) return rc;
  std::unique_ptr<pyr3_renderer> r(new pyr3_renderer());
  r->device = opts->device;
  CUDA_TRY(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
  CUDA_TRY(cudaEventCreate(&r->ev0));
  CUDA_TRY(cudaEventCreate(&r->ev1));
  for (auto& e : r->tune) CUDA_TRY(cudaEventCreate(&e));
  CUDA_TRY(cudaMalloc(&r->d_pal, 1024 * 4));
  CUDA_TRY(cudaMemsetAsync(r->d_pal, 0, 1024 * 4, r->stream));
  CUDA_TRY(cudaMalloc(&r->d_knorm, 257 * 4));
  CUDA_TRY(cudaMalloc(&r->d_kwtab, pyr3::kw_table_floats() * 4));
  CUDA_TRY(cudaMalloc(&r->d_kern, pyr3::kMaxTaps * 4));
  CUDA_TRY(cudaMalloc(&r->d_curves, 5 * 256 * 4));
  CUDA_TRY(cudaMalloc(&r->d_counters, 16));
  CUDA_TRY(cudaMemsetAsync(r->d_counters, 0, 16, r->stream));
  CUDA_TRY(cudaMalloc(&r->d_sched, 16));
  CUDA_TRY(cudaMemsetAsync(r->d_sched, 0, 16, r->stream));
  CUDA_TRY(cudaMalloc(&r->d_luma, 8));
  CUDA_TRY(cudaHostAlloc(&r->h_luma, 8, cudaHostAllocDefault));
  float knorm[257];
  kernel_norm_lut(knorm);
  CUDA_TRY(cudaMemcpyAsync(r->d_knorm, knorm, sizeof knorm, cudaMemcpyHostToDevice, r->stream));
  CUDA_TRY(pyr3::build_kw_table(r->d_knorm, r->d_kwtab, r->stream));
  rc = alloc_buffers(r.get(), opts);
  if (rc) {
    free_buffers(r.get());
    return rc;
  }
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  *out = r.release();
  return PYR3_OK;
}

PYR3_API int pyr3_destroy(pyr3_renderer* r) {
  if (!r) return PYR3_OK;
  cudaSetDevice(r->device);
  if (r->stream) cudaStreamSynchronize(r->stream);
  free_buffers(r);
  cudaFree(r->d_pal);
  cudaFree(r->d_knorm);
  cudaFree(r->d_kwtab);
  cudaFree(r->d_kern);
  cudaFree(r->d_curves);
  cudaFree(r->d_pick);
  cudaFree(r->d_counters);
  cudaFree(r->d_sched);
  cudaFree(r->d_luma);
  cudaFreeHost(r->h_luma);
  cudaFree(r->d_wrec);
  cudaFree(r->d_wave);
  cudaFree(r->d_flush);
  for (auto& e : r->marks)
    if (e) cudaEventDestroy(e);
  for (auto& e : r->tune)
    if (e) cudaEventDestroy(e);
  if (r->ev0) cudaEventDestroy(r->ev0);
  if (r->ev1) cudaEventDestroy(r->ev1);
  if (r->wave_fork) cudaEventDestroy(r->wave_fork);
  if (r->wave_join) cudaEventDestroy(r->wave_join);
  if (r->wave_aux) cudaStreamDestroy(r->wave_aux);
  if (r->stream) cudaStreamDestroy(r->stream);
  delete r;
  return PYR3_OK;
}

PYR3_API int pyr3_resize(pyr3_renderer* r, const pyr3_opts* o) {
  if (!r || !o) return fail(PYR3_E_INVALID, "null argument");
  const float fr = o->filter_radius > 0 ? o->filter_radius : 0.5f;
  if (o->width == r->W && o->height == r->H && o->oversample == r->os && fr == r->filter_radius)
    return PYR3_OK;
  int rc = set_device(r->device);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  free_buffers(r);
  return alloc_buffers(r, o);
}

PYR3_API int pyr3_reset(pyr3_renderer* r, const float* palette) {
  if (!r) return fail(PYR3_E_INVALID, "null renderer");
  cudaSetDevice(r->device);
  if (palette)
    CUDA_TRY(cudaMemcpyAsync(r->d_pal, palette, 1024 * 4, cudaMemcpyHostToDevice, r->stream));
  const size_t n = (size_t)r->SW * r->SH;
  CUDA_TRY(cudaMemsetAsync(r->d_hist, 0, n * 16, r->stream));
  CUDA_TRY(cudaMemsetAsync(r->d_idx, 0, n * 4, r->stream));
  CUDA_TRY(cudaMemsetAsync(r->d_counters, 0, 16, r->stream));
  CUDA_TRY(cudaMemsetAsync(r->d_sched, 0, 16, r->stream));
  return PYR3_OK;
}

PYR3_API int pyr3_set_capture_index(pyr3_renderer* r, int32_t on) {
  if (!r) return fail(PYR3_E_INVALID, "null renderer");
  r->capture = on != 0;
  return PYR3_OK;
}

// ---------------------------------------------------------------- iterate
static int prepare_module(pyr3_renderer* r, const pyr3_genome* g, bool aggregate,
                          std::shared_ptr<pyr3::ChaosModule>* mod) {
  if (!g || !g->xforms) return fail(PYR3_E_INVALID, "null genome");
  pyr3::GenomeShape shape;
  std::string e = pyr3::shape_from_packed(g->xforms, (int)g->n_xforms, g->final_slot, &shape);
  if (!e.empty())
    return fail(e.find("not implemented") != std::string::npos ? PYR3_E_UNSUPPORTED : PYR3_E_INVALID, e);
  std::string err;
  int rc = pyr3::get_chaos_module(shape, kWpb, aggregate, mod, &err);
  if (rc) return fail(rc, err);
  if (r && std::find(r->modules.begin(), r->modules.end(), *mod) == r->modules.end())
    r->modules.push_back(*mod);
  return PYR3_OK;
}

PYR3_API int pyr3_prepare(pyr3_renderer* r, const pyr3_genome* g) {
  if (r) cudaSetDevice(r->device);
  std::shared_ptr<pyr3::ChaosModule> m;
  return prepare_module(r, g, false, &m);
}

namespace {
// Launch one chaos kernel for `total` post-fuse samples on walkers
// walker_base.. of this launch's seed: `walkers` of them (0: pool_walkers),
// total / walkers iterations each plus one for the first total % walkers.
// Returns the walkers used through *used.
// Walkers a launch of `total` samples uses on one kernel: enough to fill
// the machine, not so many that the per-walker burn-in dominates.
uint64_t pool_walkers(pyr3_renderer* r, const pyr3::ChaosModule& m, bool queue, uint64_t total) {
  const int sms = device_sms(r->device);
  const uint64_t ctas = (uint64_t)(queue ? m.queue_blocks_per_sm : m.blocks_per_sm) * sms;
  const uint64_t per_cta = queue ? (uint64_t)pyr3::kQueueSlots : (uint64_t)m.wpb;
  const uint64_t want = std::max<uint64_t>((uint64_t)sms * 256u, total / (5ull * kFuse));
  return std::max<uint64_t>(1, std::min<uint64_t>(ctas * per_cta, std::min<uint64_t>(want, total)));
}

// The queue kernel's walker records (one slot set per resident CTA).
int queue_reserve(pyr3_renderer* r, const pyr3::ChaosModule& m) {
  const size_t rec_bytes = (size_t)m.queue_blocks_per_sm * device_sms(r->device) *
                           pyr3::kQueueSlots * pyr3::kWalkerRecordBytes;
  if (rec_bytes > r->wrec_cap) {
    CUDA_TRY(cudaStreamSynchronize(r->stream));
    cudaFree(r->d_wrec);
    r->d_wrec = nullptr;
    r->wrec_cap = 0;
    CUDA_TRY(cudaMalloc(&r->d_wrec, rec_bytes));
    r->wrec_cap = rec_bytes;
  }
  return PYR3_OK;
}

int launch_chaos(pyr3_renderer* r, const pyr3::ChaosModule& m, bool queue, ChaosArgs A,
                 uint64_t total, uint64_t walker_base, uint64_t walkers, uint64_t* used) {
  const int sms = device_sms(r->device);
  const uint64_t ctas = (uint64_t)(queue ? m.queue_blocks_per_sm : m.blocks_per_sm) * sms;
  const uint64_t per_cta = queue ? (uint64_t)pyr3::kQueueSlots : (uint64_t)m.wpb;
  const uint64_t nw = walkers ? walkers : pool_walkers(r, m, queue, total);
  const uint64_t base = total / nw, extra = total % nw;
  if (queue && base + 1 + kFuse > 0xffffffffull)
    return fail(PYR3_E_INVALID, "too many iterations per walker for one launch (> 2^32)");
  A.walker_base = walker_base;
  A.n_walkers = nw;
  A.iters_base = base;
  A.iters_extra = extra;
  void* params[] = {&A};
  if (queue) {
    // One persistent CTA per SM; each fills cta_slots of its slots first
    // (fewer than all for small launches, so the walkers spread over every
    // SM) and refills slots from sched[0] as walkers finish.
    const int rc = queue_reserve(r, m);
    if (rc) return rc;
    uint64_t slots = (nw + ctas - 1) / ctas;
    slots = std::min<uint64_t>(per_cta, (slots + 31) & ~31ull);
    A.wrec = r->d_wrec;
    A.cta_slots = (uint32_t)slots;
    CUDA_TRY(cudaMemsetAsync(r->d_sched, 0, 8, r->stream));
    LAUNCH_TRY(m.queue, (unsigned)ctas, (unsigned)(pyr3::kQueueWarps * 32), m.queue_smem, r->stream,
               params);
    r->last_launches += 1;
  } else {
    const unsigned grid = (unsigned)std::min<uint64_t>((nw + m.wpb - 1) / m.wpb, ctas);
    LAUNCH_TRY(m.chaos, grid, (unsigned)m.wpb, m.smem, r->stream, params);
    r->last_launches += 1;
  }
  *used = nw;
  return PYR3_OK;
}

// Most walkers one wave launch takes (a caller's explicit count): their
// state (49 u32 per walker and region, two buffers) stays within a few GB.
constexpr uint64_t kWaveMaxWalkers = 1ull << 21;
// Walkers of a wave launch: total / 2000 for large launches (2,000
// iterations each), but no more than the walkers whose state fills half of
// L2, so a walker's record, written at the end of one iteration, is still
// in L2 when the next launch of its population copies it in (the copy then
// drops the lines, see chaos_wave_kernel); at least enough to fill the GPU
// twice over (two populations) -- but a small launch takes only
// sqrt(1200 * total), since every walker also runs the 200-iteration
// burn-in: measured on B200 at 2e6, 9.4e6 and 3.4e7 samples, that is within
// 5 % of the best walker count, where the fill alone was 7-38 % slower.
// On the headline genome (1.04e9 samples) pools of 227 K-346 K walkers run
// within 2 % of each other and 15 % faster than 518 K, whose state spills
// to HBM.
uint64_t wave_walkers(pyr3_renderer* r, const pyr3::ChaosModule& m, uint64_t total) {
  const uint64_t wb2 = 2ull * pyr3::kWaveBlock;
  const uint64_t fill = (uint64_t)device_sms(r->device) * (uint64_t)m.wave_blocks_per_sm * wb2;
  const uint64_t l2 = std::max<uint64_t>(fill, device_l2(r->device) / 2 / (pyr3::kWaveFields * 4) / wb2 * wb2);
  const uint64_t small = (uint64_t)std::sqrt(1200.0 * (double)total);
  const uint64_t want = std::max<uint64_t>(std::min<uint64_t>(fill, small), std::min<uint64_t>(l2, total / 2000));
  return std::max<uint64_t>(1, std::min<uint64_t>(want, total));
}

// The wave kernel for `total` samples on walkers walker_base.. (`walkers`
// of them, 0: wave_walkers).  The walkers are split into two populations,
// each with its own state and launch sequence on its own stream: a seeding
// launch, one launch per iteration (the iterations of its longest walker,
// fuse included), and a last launch that finishes the walkers whose
// bad-value retries did not count as iterations.  The two sequences
// interleave, so one population's blocks fill the SMs while the other's
// launch drains its last blocks (and across the gap between launches).
// The walkers, their streams and iteration counts are those of one
// population of `walkers`, so the histogram is the same.
constexpr int kWavePops = 2;
struct WavePlan {
  int pops = 1;
  uint64_t first[kWavePops] = {}, n[kWavePops] = {}, cap[kWavePops] = {};
  size_t off[kWavePops] = {};  // u32 offset of each population's block in d_wave
};

// Split nw walkers into populations and make sure the state buffer and the
// second stream exist.  Each population's block (two state buffers, then
// its 3 x NXF counts) starts on a 256-byte boundary, so every chunk field
// the bulk copies read is 1 KB aligned.
int wave_reserve(pyr3_renderer* r, const pyr3::ChaosModule& m, uint64_t nw, WavePlan* plan) {
  if (nw > kWaveMaxWalkers) return fail(PYR3_E_INVALID, "wave kernel: more than 2^21 walkers");
  const uint64_t wb = pyr3::kWaveBlock;
  const size_t nxf = (size_t)m.nxf;
  plan->pops = nw >= 2 * wb ? kWavePops : 1;
  size_t bytes = 0;
  for (int p = 0; p < plan->pops; ++p) {
    plan->first[p] = p == 0 ? 0 : plan->first[p - 1] + plan->n[p - 1];
    plan->n[p] = p + 1 == plan->pops ? nw - plan->first[p] : (nw / plan->pops + wb - 1) / wb * wb;
    plan->cap[p] = (plan->n[p] + wb - 1) / wb * wb;
    plan->off[p] = bytes / 4;
    const size_t blk = (2 * nxf * pyr3::kWaveFields * plan->cap[p] + 3 * nxf) * 4;
    bytes += (blk + 255) / 256 * 256;
  }
  if (bytes > r->wave_bytes) {
    CUDA_TRY(cudaStreamSynchronize(r->stream));
    cudaFree(r->d_wave);
    r->d_wave = nullptr;
    r->wave_bytes = 0;
    CUDA_TRY(cudaMalloc(&r->d_wave, bytes));
    r->wave_bytes = bytes;
  }
  if (plan->pops > 1 && !r->wave_aux) {
    CUDA_TRY(cudaStreamCreateWithFlags(&r->wave_aux, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreateWithFlags(&r->wave_fork, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&r->wave_join, cudaEventDisableTiming));
  }
  return PYR3_OK;
}

int launch_wave(pyr3_renderer* r, const pyr3::ChaosModule& m, const ChaosArgs& A0, uint64_t total,
                uint64_t walker_base, uint64_t walkers, uint64_t* used) {
  const uint64_t nw = walkers ? walkers : wave_walkers(r, m, total);
  const uint64_t base = total / nw, extra = total % nw;
  if (base + 1 + kFuse > 0xffffffffull)
    return fail(PYR3_E_INVALID, "too many iterations per walker for one launch (> 2^32)");
  const uint64_t wb = pyr3::kWaveBlock;
  const size_t nxf = (size_t)m.nxf;
  WavePlan plan;
  int rc = wave_reserve(r, m, nw, &plan);
  if (rc) return rc;
  const int pops = plan.pops;
  cudaStream_t st[kWavePops] = {r->stream, r->wave_aux};
  if (pops > 1) {
    CUDA_TRY(cudaEventRecord(r->wave_fork, r->stream));
    CUDA_TRY(cudaStreamWaitEvent(r->wave_aux, r->wave_fork, 0));
  }
  ChaosArgs A[kWavePops];
  WaveArgs W[kWavePops];
  uint64_t steps[kWavePops] = {}, max_steps = 0;
  unsigned grid[kWavePops] = {};
  for (int p = 0; p < pops; ++p) {
    A[p] = A0;
    A[p].walker_base = walker_base + plan.first[p];
    A[p].n_walkers = plan.n[p];
    A[p].iters_base = base;
    A[p].iters_extra =
        extra > plan.first[p] ? std::min<uint64_t>(extra - plan.first[p], plan.n[p]) : 0;
    std::memset(&W[p], 0, sizeof W[p]);
    W[p].st = r->d_wave + plan.off[p];
    W[p].cnt = W[p].st + 2 * nxf * pyr3::kWaveFields * plan.cap[p];
    W[p].cap = plan.cap[p];
    CUDA_TRY(cudaMemsetAsync(W[p].cnt, 0, 3 * nxf * 4, st[p]));
    W[p].mode = 0;
    W[p].rd_buf = 1;
    W[p].wr_buf = 0;
    W[p].rd_cnt = 2;
    W[p].wr_cnt = 0;
    W[p].zero_cnt = 1;
    void* params[] = {&A[p], &W[p]};
    const unsigned seed_grid = (unsigned)((plan.n[p] + wb - 1) / wb);
    LAUNCH_TRY(m.wave, seed_grid, (unsigned)wb, m.wave_smem, st[p], params);
    r->last_launches += 1;
    grid[p] = seed_grid + (unsigned)nxf;  // >= chunks of any split into regions
    steps[p] = base + (A[p].iters_extra ? 1 : 0) + kFuse;
    max_steps = std::max(max_steps, steps[p]);
  }
  for (uint64_t s = 1; s <= max_steps + 1; ++s) {
    for (int p = 0; p < pops; ++p) {
      if (s > steps[p] + 1) continue;
      W[p].mode = s <= steps[p] ? 1u : 2u;
      W[p].rd_buf = (uint32_t)((s - 1) & 1);
      W[p].wr_buf = W[p].rd_buf ^ 1u;
      W[p].rd_cnt = (uint32_t)((s - 1) % 3);
      W[p].wr_cnt = (uint32_t)(s % 3);
      W[p].zero_cnt = (uint32_t)((s + 1) % 3);
      void* params[] = {&A[p], &W[p]};
      LAUNCH_TRY(m.wave, grid[p], (unsigned)wb, m.wave_smem, st[p], params);
      r->last_launches += 1;
    }
  }
  if (pops > 1) {
    CUDA_TRY(cudaEventRecord(r->wave_join, r->wave_aux));
    CUDA_TRY(cudaStreamWaitEvent(r->stream, r->wave_join, 0));
  }
  *used = nw;
  return PYR3_OK;
}

enum KernelKind { kBarrier = 0, kQueue = 1, kWave = 2 };

// Walkers a launch of `total` samples uses on kernel `kind` by default.
uint64_t kind_walkers(pyr3_renderer* r, const pyr3::ChaosModule& m, int kind, uint64_t total) {
  return kind == kWave ? wave_walkers(r, m, total) : pool_walkers(r, m, kind == kQueue, total);
}

int launch_kind(pyr3_renderer* r, const pyr3::ChaosModule& m, int kind, const ChaosArgs& A,
                uint64_t total, uint64_t walker_base, uint64_t walkers, uint64_t* used) {
  if (kind == kWave) return launch_wave(r, m, A, total, walker_base, walkers, used);
  return launch_chaos(r, m, kind == kQueue, A, total, walker_base, walkers, used);
}
}  // namespace

namespace {
// Upload a genome's pick-table boundaries (renderer-owned buffer) and its
// packed xform records (the module's constant bank), on the renderer's
// stream.
int upload_genome(pyr3_renderer* r, const pyr3_genome* g, pyr3::ChaosModule& m) {
  const int n = (int)g->n_xforms;
  const bool has_final = g->final_slot >= 0;
  std::vector<float> weights(n);
  for (int i = 0; i < n; ++i) weights[i] = g->xforms[(size_t)i * 116 + 3];
  std::vector<uint16_t> starts;
  std::string err;
  if (!build_pick_starts(n, weights.data(), g->xaos, &starts, &err)) return fail(PYR3_E_INVALID, err);
  const size_t pick_bytes = starts.size() * 2;
  if (r->pick_cap < pick_bytes) {
    CUDA_TRY(cudaStreamSynchronize(r->stream));
    cudaFree(r->d_pick);
    r->d_pick = nullptr;
    CUDA_TRY(cudaMalloc(&r->d_pick, std::max<size_t>(pick_bytes, 4096)));
    r->pick_cap = std::max<size_t>(pick_bytes, 4096);
  }
  CUDA_TRY(cudaMemcpyAsync(r->d_pick, starts.data(), pick_bytes, cudaMemcpyHostToDevice, r->stream));
  const size_t xf_bytes = (size_t)(n + (has_final ? 1 : 0)) * 116 * 4;
  if (xf_bytes > m.c_xf_bytes) return fail(PYR3_E_INVALID, "xform records exceed module constant bank");
  CUDA_TRY(cudaMemcpyAsync(m.c_xf, g->xforms, xf_bytes, cudaMemcpyHostToDevice, r->stream));
  return PYR3_OK;
}

// Launch arguments of a chaos kernel that do not depend on the walker split
// (chaos uniforms, src/chaos.ts:381-456).
ChaosArgs base_args(pyr3_renderer* r, const pyr3_genome* g, const pyr3_iterate_opts* o) {
  ChaosArgs A;
  std::memset(&A, 0, sizeof A);
  A.hist = r->d_hist;
  A.idx_sum = r->capture ? r->d_idx : nullptr;
  A.palette = r->d_pal;
  A.pick_start = r->d_pick;
  A.fuse = kFuse;
  A.width = r->SW;
  A.height = r->SH;
  A.scale = (float)((double)g->scale * (double)r->os);
  A.cx = g->cx;
  A.cy = g->cy;
  const float rot = (float)(((double)g->rotate_deg * M_PI) / 180.0);
  A.cos_r = std::cos(rot);
  A.sin_r = std::sin(rot);
  A.seed = o->seed;
  A.jitter = o->walker_jitter >= 0.0f ? o->walker_jitter : kDefaultJitter;
  A.palette_mode = g->palette_mode;
  A.capture_index = r->capture ? 1u : 0u;
  A.color_mode = o->color_mode;
  A.flow_strength = o->flow_strength;
  A.flow_scale = o->flow_scale;
  A.trap_kind = o->trap_kind;
  A.trap_mode = o->trap_mode;
  A.trap_cx = o->trap_cx;
  A.trap_cy = o->trap_cy;
  A.trap_radius = o->trap_radius;
  const double ta = (double)o->trap_angle_deg * M_PI / 180.0;
  A.trap_nx = (float)-std::sin(ta);
  A.trap_ny = (float)std::cos(ta);
  A.trap_falloff = o->trap_falloff;
  A.trap_freq = o->trap_freq;
  A.trap_strength = o->trap_strength;
  A.phase_strength = o->phase_strength;
  A.phase_freq = o->phase_freq;
  A.xform_blend = std::min(1.0f, std::max(0.0f, g->xform_blend));
  A.counters = r->d_counters;
  A.sched = r->d_sched;

  return A;
}
}  // namespace

PYR3_API int pyr3_iterate(pyr3_renderer* r, const pyr3_genome* g, const pyr3_iterate_opts* o) {
  if (!r || !g || !o) return fail(PYR3_E_INVALID, "null argument");
  cudaSetDevice(r->device);
  const bool aggregate = (o->flags & PYR3_ITER_AGGREGATE) != 0;
  std::shared_ptr<pyr3::ChaosModule> m;
  int rc = prepare_module(r, g, aggregate, &m);
  if (rc) return rc;
  rc = upload_genome(r, g, *m);
  if (rc) return rc;
  const uint64_t total = o->walkers * o->iters_per_walker;
  if (total == 0) return PYR3_OK;
  ChaosArgs A = base_args(r, g, o);

  const bool exact = (o->flags & PYR3_ITER_EXACT_WALKERS) != 0;
  uint64_t done = 0, walker_base = 0, used = 0;
  const bool wave_ok = m->wave && (!exact || o->walkers <= kWaveMaxWalkers);
  int kind = kBarrier;
  r->last_launches = 0;
  CUDA_TRY(cudaEventRecord(r->ev0, r->stream));
  if (o->flags & PYR3_ITER_KERNEL_BARRIER) {
    kind = kBarrier;
  } else if (o->flags & PYR3_ITER_KERNEL_QUEUE) {
    kind = m->queue ? kQueue : kBarrier;
  } else if (o->flags & PYR3_ITER_KERNEL_WAVE) {
    kind = wave_ok ? kWave : kBarrier;
  } else if (m->choice.load() >= 0) {
    kind = m->choice.load();
    if ((kind == kQueue && !m->queue) || (kind == kWave && !wave_ok)) kind = kBarrier;
  } else if (!exact && total >= kTuneMinSamples) {
    // Autotune: the first large launch of this genome structure runs a
    // short trial on each chaos kernel -- with the walker count that kernel
    // would use for the whole launch, so that the trial sees the same
    // occupancy and queue lengths -- and the rest of the samples (and every
    // later launch) on the kernel whose predicted time for the remaining
    // samples, burn-in included, is lowest.  Every sample still lands in the
    // histogram; each launch uses fresh walker indices.
    int cand[3];
    int nc = 0;
    cand[nc++] = kBarrier;
    if (m->queue) cand[nc++] = kQueue;
    if (m->wave) cand[nc++] = kWave;
    uint64_t nw[3], tr[3];
    float ms[3];
    // Buffers first, so no trial's time includes an allocation.
    for (int c = 0; c < nc; ++c) {
      nw[c] = kind_walkers(r, *m, cand[c], total);
      if (cand[c] == kQueue) rc = queue_reserve(r, *m);
      if (cand[c] == kWave) {
        WavePlan plan;
        rc = wave_reserve(r, *m, nw[c], &plan);
      }
      if (rc) return rc;
    }
    CUDA_TRY(cudaEventRecord(r->tune[0], r->stream));
    for (int c = 0; c < nc; ++c) {
      tr[c] = nw[c] * std::max<uint64_t>(1, total / 32 / nw[c]);
      rc = launch_kind(r, *m, cand[c], A, tr[c], walker_base, nw[c], &used);
      if (rc) return rc;
      walker_base += used;
      done += tr[c];
      CUDA_TRY(cudaEventRecord(r->tune[c + 1], r->stream));
    }
    CUDA_TRY(cudaEventSynchronize(r->tune[nc]));
    const double rest = (double)(total > done ? total - done : 0);
    double best = 0.0;
    for (int c = 0; c < nc; ++c) {
      CUDA_TRY(cudaEventElapsedTime(&ms[c], r->tune[c], r->tune[c + 1]));
      // ms per iteration (burn-in iterations included) times the
      // iterations the rest of the launch needs on this kernel.
      const double per = ms[c] / ((double)tr[c] + (double)nw[c] * kFuse);
      const double pred = per * (rest + (double)kind_walkers(r, *m, cand[c], total) * kFuse);
      if (c == 0 || pred < best) {
        best = pred;
        kind = cand[c];
      }
    }
    m->choice.store(kind);
  }
  if (done < total) {
    if (exact) rc = launch_kind(r, *m, kind, A, total, 0, o->walkers, &used);
    else rc = launch_kind(r, *m, kind, A, total - done, walker_base, 0, &used);
    if (rc) return rc;
  }
  CUDA_TRY(cudaEventRecord(r->ev1, r->stream));
  return PYR3_OK;
}

PYR3_API int pyr3_last_iterate_launches(pyr3_renderer* r, uint64_t* launches) {
  if (!r || !launches) return fail(PYR3_E_INVALID, "null argument");
  *launches = r->last_launches;
  return PYR3_OK;
}

PYR3_API int pyr3_last_iterate_ms(pyr3_renderer* r, float* ms) {
  if (!r || !ms) return fail(PYR3_E_INVALID, "null argument");
  CUDA_TRY(cudaEventSynchronize(r->ev1));
  CUDA_TRY(cudaEventElapsedTime(ms, r->ev0, r->ev1));
  return PYR3_OK;
}

// ------------------------------------------------------------------ batch
// Many renderers, each with its own genome and iterate request, rendered by
// one CUDA graph: every genome gets its own instance of its specialised
// module (its own constant bank, so genomes of one structure do not collide)
// and the graph clears each renderer's histogram and runs each genome's
// chaos kernel, spread over worker streams so the launches run
// concurrently.  Walkers per genome are chosen for the batch: enough
// iterations per walker to keep the 200-iteration burn-in under ~10 %,
// since the GPU is filled by running many genomes at once.
//
// Genomes large enough to fill the GPU on their own (at least
// kBatchSoloSamples, pooled walkers) stay out of the graph: each
// runs through pyr3_iterate on its autotuned kernel, one after another on
// their renderers' streams, while the graph runs the small ones.  Their
// genome records are copied at creation.  Graph genomes use module
// instances 1.., so they never share a constant bank with pyr3_iterate's
// instance 0.
struct pyr3_batch {
  int device = 0;
  cudaStream_t origin = nullptr;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
  std::vector<std::shared_ptr<pyr3::ChaosModule>> mods;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t samples = 0;
  // Genomes run through pyr3_iterate, with their own copies of the records.
  std::vector<pyr3_renderer*> solo_r;
  std::vector<pyr3_genome> solo_g;
  std::vector<pyr3_iterate_opts> solo_o;
  std::vector<std::vector<float>> solo_xf, solo_xaos;
  std::vector<cudaEvent_t> solo_ev;
  // Every distinct renderer of the batch, cleared once per run, and the
  // event after those clears.
  std::vector<pyr3_renderer*> clear_r;
  cudaEvent_t cleared = nullptr;
  // Pick tables of the graph genomes (one device buffer each, so genomes
  // that share a renderer keep their own).
  std::vector<uint16_t*> picks;
};

namespace {
constexpr uint64_t kBatchItersPerWalker = 2000;
// A small genome may take more walkers, down to this many iterations each
// (the 200-iteration burn-in is then a quarter of its work), so that the
// batch's concurrent kernels together fill the GPU.
constexpr uint64_t kBatchMinItersPerWalker = 600;
// Measured on the 256-genome batch: run alone, one after another, every
// genome of 2^24 samples or more beats sharing the GPU with the graph.
constexpr uint64_t kBatchSoloSamples = 1ull << 24;

void free_batch(pyr3_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto s : b->streams) cudaStreamDestroy(s);
  for (auto e : b->joins) cudaEventDestroy(e);
  for (auto e : b->solo_ev) cudaEventDestroy(e);
  for (auto p : b->picks) cudaFree(p);
  if (b->cleared) cudaEventDestroy(b->cleared);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->origin) cudaStreamDestroy(b->origin);
  delete b;
}
}  // namespace

PYR3_API int pyr3_batch_create(pyr3_renderer* const* renderers, const pyr3_genome* genomes,
                               const pyr3_iterate_opts* opts, uint32_t n, uint32_t n_streams,
                               pyr3_batch** out) {
  if (!renderers || !genomes || !opts || !out || n == 0 || n_streams == 0)
    return fail(PYR3_E_INVALID, "bad arguments");
  const int dev = renderers[0] ? renderers[0]->device : 0;
  for (uint32_t i = 0; i < n; ++i)
    if (!renderers[i] || renderers[i]->device != dev)
      return fail(PYR3_E_INVALID, "batch renderers must be non-null and on one device");
  cudaSetDevice(dev);
  std::unique_ptr<pyr3_batch, void (*)(pyr3_batch*)> b(new pyr3_batch(), free_batch);
  b->device = dev;
  CUDA_TRY(cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking));
  CUDA_TRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&b->cleared, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreate(&b->ev0));
  CUDA_TRY(cudaEventCreate(&b->ev1));
  const uint32_t k = std::min(n_streams, n);
  for (uint32_t j = 0; j < k; ++j) {
    cudaStream_t st;
    cudaEvent_t ev;
    CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    b->streams.push_back(st);
    CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    b->joins.push_back(ev);
  }
  // Modules (one instance per genome of a repeated structure), tables and
  // records, and the launch arguments.
  std::map<std::string, int> seen;
  std::vector<ChaosArgs> args;
  std::vector<unsigned> grids;
  std::vector<pyr3_renderer*> graph_r;
  const int sms = device_sms(dev);
  for (uint32_t i = 0; i < n; ++i)
    if (std::find(b->clear_r.begin(), b->clear_r.end(), renderers[i]) == b->clear_r.end())
      b->clear_r.push_back(renderers[i]);
  // Compile every genome structure not in the cubin cache yet, in parallel
  // on the host, before the modules load one by one below.
  {
    std::vector<pyr3::GenomeShape> shapes;
    std::vector<bool> agg;
    for (uint32_t i = 0; i < n; ++i) {
      pyr3::GenomeShape shape;
      if (genomes[i].xforms &&
          pyr3::shape_from_packed(genomes[i].xforms, (int)genomes[i].n_xforms, genomes[i].final_slot, &shape)
              .empty()) {
        shapes.push_back(std::move(shape));
        agg.push_back((opts[i].flags & PYR3_ITER_AGGREGATE) != 0);
      }
    }
    pyr3::precompile_chaos(shapes, agg, kWpb);
  }
  for (uint32_t i = 0; i < n; ++i) {
    pyr3_renderer* r = renderers[i];
    const pyr3_genome* g = &genomes[i];
    const pyr3_iterate_opts* o = &opts[i];
    if (!g->xforms) return fail(PYR3_E_INVALID, "null genome in batch");
    pyr3::GenomeShape shape;
    std::string e = pyr3::shape_from_packed(g->xforms, (int)g->n_xforms, g->final_slot, &shape);
    if (!e.empty())
      return fail(e.find("not implemented") != std::string::npos ? PYR3_E_UNSUPPORTED : PYR3_E_INVALID, e);
    const uint64_t total = o->walkers * o->iters_per_walker;
    if (!(o->flags & PYR3_ITER_EXACT_WALKERS) && total >= kBatchSoloSamples) {
      const size_t nrec = (size_t)g->n_xforms + (g->final_slot >= 0 ? 1 : 0);
      b->solo_xf.emplace_back(g->xforms, g->xforms + nrec * 116);
      b->solo_xaos.emplace_back();
      if (g->xaos) b->solo_xaos.back().assign(g->xaos, g->xaos + (size_t)g->n_xforms * g->n_xforms);
      b->solo_r.push_back(r);
      b->solo_g.push_back(*g);
      b->solo_o.push_back(*o);
      cudaEvent_t ev;
      CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      b->solo_ev.push_back(ev);
      b->samples += total;
      continue;
    }
    const bool aggregate = (o->flags & PYR3_ITER_AGGREGATE) != 0;
    const std::string key = shape.key() + (aggregate ? "|A" : "");
    const int inst = 1 + seen[key]++;
    std::shared_ptr<pyr3::ChaosModule> m;
    std::string err;
    int rc = pyr3::get_chaos_module(shape, kWpb, aggregate, &m, &err, inst);
    if (rc) return fail(rc, err);
    b->mods.push_back(m);
    // This genome's own pick table; its xform records go to its module
    // instance's constant bank.
    {
      const int nx = (int)g->n_xforms;
      std::vector<float> weights(nx);
      for (int x = 0; x < nx; ++x) weights[x] = g->xforms[(size_t)x * 116 + 3];
      std::vector<uint16_t> starts;
      std::string perr;
      if (!build_pick_starts(nx, weights.data(), g->xaos, &starts, &perr)) return fail(PYR3_E_INVALID, perr);
      uint16_t* pk = nullptr;
      CUDA_TRY(cudaMalloc(&pk, starts.size() * 2));
      b->picks.push_back(pk);
      CUDA_TRY(cudaMemcpy(pk, starts.data(), starts.size() * 2, cudaMemcpyHostToDevice));
      const size_t xf_bytes = (size_t)(nx + (g->final_slot >= 0 ? 1 : 0)) * 116 * 4;
      if (xf_bytes > m->c_xf_bytes) return fail(PYR3_E_INVALID, "xform records exceed module constant bank");
      CUDA_TRY(cudaMemcpy(m->c_xf, g->xforms, xf_bytes, cudaMemcpyHostToDevice));
    }
    ChaosArgs A = base_args(r, g, o);
    A.pick_start = b->picks.back();
    uint64_t nw;
    if (o->flags & PYR3_ITER_EXACT_WALKERS) {
      nw = std::max<uint64_t>(1, o->walkers);
    } else {
      const uint64_t cap = (uint64_t)m->blocks_per_sm * sms * m->wpb;
      // One kernel per stream runs at a time: each gets its share of the
      // GPU's resident blocks, as far as its samples allow.
      const uint64_t fill = ((uint64_t)m->blocks_per_sm * sms + k - 1) / k * m->wpb;
      const uint64_t want = std::max<uint64_t>(std::max<uint64_t>(256, total / kBatchItersPerWalker),
                                               std::min<uint64_t>(fill, total / kBatchMinItersPerWalker));
      nw = std::max<uint64_t>(1, std::min<uint64_t>(cap, want));
      nw = std::min<uint64_t>(nw, std::max<uint64_t>(1, total));
    }
    A.walker_base = 0;
    A.n_walkers = nw;
    A.iters_base = total / nw;
    A.iters_extra = total % nw;
    args.push_back(A);
    grids.push_back((unsigned)std::min<uint64_t>((nw + m->wpb - 1) / m->wpb, (uint64_t)m->blocks_per_sm * sms));
    graph_r.push_back(r);
    b->samples += total;
  }
  // Pointers into the copies are taken once every copy is in place.
  for (size_t s = 0; s < b->solo_g.size(); ++s) {
    b->solo_g[s].xforms = b->solo_xf[s].data();
    b->solo_g[s].xaos = b->solo_xaos[s].empty() ? nullptr : b->solo_xaos[s].data();
  }
  const uint32_t ng = (uint32_t)graph_r.size();
  // Capture: fork to the worker streams, each genome's chaos kernel, join
  // back.  (The clears run before the graph, in pyr3_batch_run.)
  CUDA_TRY(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
  cudaError_t ce = cudaEventRecord(b->fork, b->origin);
  for (uint32_t j = 0; j < k && ce == cudaSuccess; ++j) ce = cudaStreamWaitEvent(b->streams[j], b->fork, 0);
  for (uint32_t i = 0; i < ng && ce == cudaSuccess; ++i) {
    pyr3_renderer* r = graph_r[i];
    (void)r;
    cudaStream_t st = b->streams[i % k];
    void* params[] = {&args[i]};
    ce = cudaLaunchKernel((const void*)b->mods[i]->chaos, dim3(grids[i]), dim3(b->mods[i]->wpb), params,
                          b->mods[i]->smem, st);
  }
  for (uint32_t j = 0; j < k && ce == cudaSuccess; ++j) {
    ce = cudaEventRecord(b->joins[j], b->streams[j]);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->origin, b->joins[j], 0);
  }
  cudaGraph_t graph = nullptr;
  cudaError_t ee = cudaStreamEndCapture(b->origin, &graph);
  if (ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return fail(PYR3_E_CUDA, std::string("batch capture: ") + cudaGetErrorString(ce));
  }
  if (ee != cudaSuccess) return fail(PYR3_E_CUDA, std::string("batch capture: ") + cudaGetErrorString(ee));
  b->graph = graph;
  CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
  *out = b.release();
  return PYR3_OK;
}

PYR3_API int pyr3_batch_run(pyr3_batch* b) {
  if (!b) return fail(PYR3_E_INVALID, "null batch");
  cudaSetDevice(b->device);
  CUDA_TRY(cudaEventRecord(b->ev0, b->origin));
  // Every distinct renderer once, so genomes that share one (the sub-frames
  // of a motion-blurred frame) all accumulate into it.
  for (pyr3_renderer* r : b->clear_r) {
    CUDA_TRY(cudaMemsetAsync(r->d_hist, 0, (size_t)r->SW * r->SH * 16, b->origin));
    CUDA_TRY(cudaMemsetAsync(r->d_counters, 0, 16, b->origin));
  }
  CUDA_TRY(cudaEventRecord(b->cleared, b->origin));
  CUDA_TRY(cudaGraphLaunch(b->exec, b->origin));
  // Large genomes: one after another (each waits for the previous one's
  // work), beside the graph.
  cudaEvent_t prev = b->cleared;
  for (size_t s = 0; s < b->solo_r.size(); ++s) {
    pyr3_renderer* r = b->solo_r[s];
    CUDA_TRY(cudaStreamWaitEvent(r->stream, prev, 0));
    const int rc = pyr3_iterate(r, &b->solo_g[s], &b->solo_o[s]);
    if (rc) return rc;
    CUDA_TRY(cudaEventRecord(b->solo_ev[s], r->stream));
    prev = b->solo_ev[s];
  }
  if (prev != b->cleared) CUDA_TRY(cudaStreamWaitEvent(b->origin, prev, 0));
  CUDA_TRY(cudaEventRecord(b->ev1, b->origin));
  return PYR3_OK;
}

PYR3_API int pyr3_batch_sync(pyr3_batch* b, float* ms, uint64_t* samples) {
  if (!b) return fail(PYR3_E_INVALID, "null batch");
  cudaSetDevice(b->device);
  CUDA_TRY(cudaEventSynchronize(b->ev1));
  if (ms) CUDA_TRY(cudaEventElapsedTime(ms, b->ev0, b->ev1));
  if (samples) *samples = b->samples;
  return PYR3_OK;
}

PYR3_API int pyr3_batch_destroy(pyr3_batch* b) {
  if (!b) return PYR3_OK;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->origin);
  free_batch(b);
  return PYR3_OK;
}

// ---------------------------------------------------------------- denoiser
// Layers of the learned denoiser's U-Net on device tensors (NCHW f32, each
// operand a pointer plus per-image stride).  Argument checks only; the
// shapes' consistency with the buffers is the caller's.
namespace {
bool dn_dims_ok(int64_t a, int64_t b, int64_t c, int64_t d) { return a > 0 && b > 0 && c > 0 && d > 0; }
}  // namespace

PYR3_API int pyr3_dn_conv3x3(const float* in, int64_t in_ns, int32_t ci, float* out, int64_t out_ns,
                             int32_t co, int32_t n, int32_t h, int32_t w, const float* weight,
                             const float* bias, int32_t relu, void* stream) {
  if (!in || !out || !weight || !dn_dims_ok(ci, co, n, (int64_t)h * w) || h <= 0 || w <= 0)
    return fail(PYR3_E_INVALID, "conv3x3: null operand or non-positive size");
  CUDA_TRY(pyr3::dn_conv3x3(in, in_ns, ci, out, out_ns, co, n, h, w, weight, bias, relu != 0,
                            (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API int pyr3_dn_conv3x3_bf16(const float* in, int64_t in_ns, int32_t ci, float* out, int64_t out_ns,
                                  int32_t co, int32_t n, int32_t h, int32_t w, const float* weight,
                                  const float* bias, int32_t relu, void* stream) {
  if (!in || !out || !weight || !dn_dims_ok(ci, co, n, (int64_t)h * w) || h <= 0 || w <= 0 || co > 128)
    return fail(PYR3_E_INVALID, "conv3x3_bf16: null operand, non-positive size or more than 128 outputs");
  CUDA_TRY(pyr3::dn_conv3x3_bf16(in, in_ns, ci, out, out_ns, co, n, h, w, weight, bias, relu != 0,
                                 (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API int pyr3_dn_conv3x3_wgrad(const float* in, int64_t in_ns, int32_t ci, const float* dout,
                                   int64_t dout_ns, int32_t co, int32_t n, int32_t h, int32_t w,
                                   float* dweight, float* dbias, float* scratch, uint64_t scratch_floats,
                                   void* stream) {
  if (!in || !dout || !dweight || !scratch || !dn_dims_ok(ci, co, n, (int64_t)h * w) || h <= 0 || w <= 0)
    return fail(PYR3_E_INVALID, "conv3x3_wgrad: null operand or non-positive size");
  if (scratch_floats < pyr3::dn_wgrad_scratch_floats(co, ci))
    return fail(PYR3_E_INVALID, "conv3x3_wgrad: scratch smaller than pyr3_dn_wgrad_scratch_floats");
  CUDA_TRY(pyr3::dn_conv3x3_wgrad(in, in_ns, ci, dout, dout_ns, co, n, h, w, dweight, dbias, scratch,
                                  (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API int pyr3_dn_conv3x3_wgrad_bf16(const float* in, int64_t in_ns, int32_t ci, const float* dout,
                                        int64_t dout_ns, int32_t co, int32_t n, int32_t h, int32_t w,
                                        float* dweight, float* dbias, float* scratch, uint64_t scratch_floats,
                                        void* stream) {
  if (!in || !dout || !dweight || !scratch || !dn_dims_ok(ci, co, n, (int64_t)h * w) || h <= 0 || w <= 0 ||
      co > 128 || ci > 128 || n > 32)
    return fail(PYR3_E_INVALID, "conv3x3_wgrad_bf16: null operand or size out of range");
  if (scratch_floats < pyr3::dn_wgrad_scratch_floats(co, ci))
    return fail(PYR3_E_INVALID, "conv3x3_wgrad_bf16: scratch smaller than pyr3_dn_wgrad_scratch_floats");
  CUDA_TRY(pyr3::dn_conv3x3_wgrad_bf16(in, in_ns, ci, dout, dout_ns, co, n, h, w, dweight, dbias, scratch,
                                       (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API uint64_t pyr3_dn_wgrad_scratch_floats(int32_t co, int32_t ci) {
  return co > 0 && ci > 0 ? (uint64_t)pyr3::dn_wgrad_scratch_floats(co, ci) : 0;
}

PYR3_API int pyr3_dn_flip_weights(const float* weight, int32_t co, int32_t ci, float* flipped,
                                  void* stream) {
  if (!weight || !flipped || co <= 0 || ci <= 0)
    return fail(PYR3_E_INVALID, "flip_weights: null operand or non-positive size");
  CUDA_TRY(pyr3::dn_flip_weights(weight, co, ci, flipped, (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API int pyr3_dn_relu_mask(float* grad, int64_t grad_ns, const float* y, int64_t y_ns, int32_t c,
                               int32_t n, int32_t hw, void* stream) {
  if (!grad || !y || !dn_dims_ok(c, n, hw, 1)) return fail(PYR3_E_INVALID, "relu_mask: bad arguments");
  CUDA_TRY(pyr3::dn_relu_mask(grad, grad_ns, y, y_ns, c, n, hw, (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API int pyr3_dn_add(float* y, int64_t y_ns, const float* x, int64_t x_ns, int32_t c, int32_t n,
                         int32_t hw, void* stream) {
  if (!y || !x || !dn_dims_ok(c, n, hw, 1)) return fail(PYR3_E_INVALID, "add: bad arguments");
  CUDA_TRY(pyr3::dn_add(y, y_ns, x, x_ns, c, n, hw, (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API int pyr3_dn_pool2(const float* in, int64_t in_ns, float* out, int64_t out_ns, int32_t c,
                           int32_t n, int32_t h, int32_t w, int32_t backward, int32_t accumulate,
                           void* stream) {
  if (!in || !out || !dn_dims_ok(c, n, h, w) || (h & 1) || (w & 1))
    return fail(PYR3_E_INVALID, "pool2: null operand, non-positive size or odd height/width");
  if (backward)
    CUDA_TRY(pyr3::dn_pool2_bwd(in, in_ns, out, out_ns, c, n, h, w, accumulate != 0, (cudaStream_t)stream));
  else
    CUDA_TRY(pyr3::dn_pool2(in, in_ns, out, out_ns, c, n, h, w, (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API int pyr3_dn_up2(const float* in, int64_t in_ns, float* out, int64_t out_ns, int32_t c,
                         int32_t n, int32_t h, int32_t w, int32_t backward, void* stream) {
  if (!in || !out || !dn_dims_ok(c, n, h, w)) return fail(PYR3_E_INVALID, "up2: bad arguments");
  if (backward)
    CUDA_TRY(pyr3::dn_up2_bwd(in, in_ns, out, out_ns, c, n, h, w, (cudaStream_t)stream));
  else
    CUDA_TRY(pyr3::dn_up2(in, in_ns, out, out_ns, c, n, h, w, (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API int pyr3_dn_mse(const float* pred, const float* target, int64_t count, float* grad,
                         float* loss_sum, void* stream) {
  if (!pred || !target || !grad || !loss_sum || count <= 0) return fail(PYR3_E_INVALID, "mse: bad arguments");
  CUDA_TRY(pyr3::dn_mse(pred, target, count, grad, loss_sum, (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API int pyr3_dn_adam(float* param, const float* grad, float* m, float* v, int64_t count, float lr,
                          float beta1, float beta2, float eps, int32_t step, void* stream) {
  if (!param || !grad || !m || !v || count <= 0 || step < 1) return fail(PYR3_E_INVALID, "adam: bad arguments");
  CUDA_TRY(pyr3::dn_adam(param, grad, m, v, count, lr, beta1, beta2, eps, step, (cudaStream_t)stream));
  return PYR3_OK;
}

// ---------------------------------------------------------------- present
// `brightness` replaces p->brightness: the auto-exposure loop presents at a
// brightness it holds in double, as the reference's genome does.
static int run_present(pyr3_renderer* r, const pyr3_present_opts* p, uint64_t total_samples,
                       void* dev_out, int32_t out_kind, double brightness) {
  if (pyr3::out_bytes_per_pixel(out_kind) == 0) return fail(PYR3_E_INVALID, "unknown output kind");
  if (total_samples == 0) return fail(PYR3_E_INVALID, "total_samples must be positive");
  // src/calibration.ts:37-43 in double, uploaded as f32.
  const double os2 = (double)r->os * (double)r->os;
  const float k1 = (float)((brightness * 255.0 * 268.0) / 256.0);
  const float k2 = (float)((os2 * p->scale * p->scale) / (255.0 * (double)total_samples));
  const float* filtered = nullptr;
  if (p->density_on) {
    int rc = ensure_filtered(r);
    if (rc) return rc;
    pyr3::DeParams d;
    d.width = r->SW;
    d.height = r->SH;
    d.max_rad = (float)((double)p->de_max_rad * r->os + 1.0);
    d.min_rad = (float)((double)p->de_min_rad * r->os + 1.0);
    d.curve = p->de_curve;
    d.k1 = k1;
    d.k2 = k2;
    d.R = (int)std::ceil(std::min(std::max(d.max_rad, 0.0f), 256.0f));
    CUDA_TRY(pyr3::launch_density(r->d_hist, r->d_filtered, d, r->d_knorm, r->d_kwtab,
                                  (unsigned long long*)(r->d_sched + 1), r->stream));
    filtered = r->d_filtered;
  }
  pyr3::TonemapParams t;
  t.width = r->W;
  t.height = r->H;
  t.oversample = r->os;
  t.fwidth = (uint32_t)r->fwidth;
  t.k1 = k1;
  t.k2 = k2;
  t.gamma = p->gamma;
  t.vibrancy = p->vibrancy;
  t.highpow = p->highpow;
  t.linrange = p->linrange;
  t.bg[0] = p->background[0];
  t.bg[1] = p->background[1];
  t.bg[2] = p->background[2];
  t.transparent = p->transparent;
  t.curves_active = p->curves ? (p->curves_active & 31u) : 0u;
  if (t.curves_active)
    CUDA_TRY(cudaMemcpyAsync(r->d_curves, p->curves, 5 * 256 * 4, cudaMemcpyHostToDevice, r->stream));
  t.hsl_active = p->hsl_active ? 1u : 0u;
  t.hsl_hue = p->hsl_hue;
  t.hsl_sat = p->hsl_sat;
  t.hsl_light = p->hsl_light;
  CUDA_TRY(pyr3::launch_tonemap(filtered ? nullptr : r->d_hist, filtered, t, r->d_kern, r->d_curves,
                                dev_out, out_kind, (unsigned long long*)(r->d_sched + 1), r->stream));
  return PYR3_OK;
}

PYR3_API int pyr3_present_device(pyr3_renderer* r, const pyr3_present_opts* p,
                                 uint64_t total_samples, void* device_out, int32_t out_kind) {
  if (!r || !p || !device_out) return fail(PYR3_E_INVALID, "null argument");
  cudaSetDevice(r->device);
  return run_present(r, p, total_samples, device_out, out_kind, p->brightness);
}

PYR3_API int pyr3_present(pyr3_renderer* r, const pyr3_present_opts* p, uint64_t total_samples,
                          void* out, int32_t out_kind) {
  if (!r || !p || !out) return fail(PYR3_E_INVALID, "null argument");
  cudaSetDevice(r->device);
  const size_t bpp = pyr3::out_bytes_per_pixel(out_kind);
  if (bpp == 0) return fail(PYR3_E_INVALID, "unknown output kind");
  const size_t bytes = (size_t)r->W * r->H * bpp;
  int rc = ensure_out(r, bytes);
  if (rc) return rc;
  rc = run_present(r, p, total_samples, r->d_out, out_kind, p->brightness);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(out, r->d_out, bytes, cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  return PYR3_OK;
}

// ------------------------------------------------------- auto-exposure
namespace {
// clamp of src/auto-exposure.ts:63-70: a non-finite value maps to lo.
double ae_clamp(double x, double lo, double hi) {
  return std::isfinite(x) ? std::min(hi, std::max(lo, x)) : lo;
}

// fitBrightnessToTarget (src/auto-exposure.ts:147-175); rerender(b, &mean)
// returns 0 or an error code that ends the fit.
template <class Rerender>
int fit_brightness(double base, double target, double initial, Rerender&& rerender,
                   pyr3_brightness_fit* fit) {
  const bool finite = std::isfinite(target) && std::isfinite(initial);
  const double factor0 = finite && initial > 0 ? target / initial : 1.0;
  *fit = pyr3_brightness_fit{base, 0, 0, initial, factor0};
  if (!finite || target <= 0 || initial <= 0 || std::fabs(factor0 - 1.0) <= PYR3_AE_DEADBAND)
    return PYR3_OK;
  double b = base, mean = initial;
  int32_t iters = 0;
  for (int k = 0; k < PYR3_AE_MAX_ITERS; ++k) {
    const double factor = target / mean;
    if (std::fabs(factor - 1.0) <= PYR3_AE_DEADBAND) break;
    b = ae_clamp(b * factor, PYR3_AE_BRIGHTNESS_MIN, PYR3_AE_BRIGHTNESS_MAX);
    const int rc = rerender(b, &mean);
    if (rc) return rc;
    ++iters;
    if (mean <= 0) break;
  }
  fit->brightness = b;
  fit->corrected = iters > 0;
  fit->iters = iters;
  fit->final_mean = mean;
  return PYR3_OK;
}

// Mean luminance of a device image on the renderer's stream: an exact
// integer sum on the device, then one division in double.
int luma_mean(pyr3_renderer* r, const void* img, uint64_t pixels, int32_t kind, double* mean) {
  if (pixels == 0) {
    *mean = 0.0;  // computeMeanLuminance: empty -> 0
    return PYR3_OK;
  }
  CUDA_TRY(cudaMemsetAsync(r->d_luma, 0, 8, r->stream));
  CUDA_TRY(pyr3::launch_luma_sum(img, pixels, kind, r->d_luma, device_sms(r->device), r->stream));
  CUDA_TRY(cudaMemcpyAsync(r->h_luma, r->d_luma, 8, cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  const double sum = (double)*r->h_luma, n = (double)pixels;
  *mean = kind == PYR3_OUT_RGBA8 ? sum / (3.0 * n) : sum * 255.0 / (3.0 * 16777216.0 * n);
  return PYR3_OK;
}
}  // namespace

PYR3_API int pyr3_fit_brightness(double base_brightness, double target_mean, double initial_mean,
                                 pyr3_rerender_fn rerender, void* ctx, pyr3_brightness_fit* fit) {
  if (!rerender || !fit) return fail(PYR3_E_INVALID, "null argument");
  return fit_brightness(base_brightness, target_mean, initial_mean,
                        [&](double b, double* mean) -> int {
                          const int rc = rerender(b, mean, ctx);
                          return rc ? fail(rc, "fit_brightness: the rerender callback failed") : PYR3_OK;
                        },
                        fit);
}

PYR3_API int pyr3_mean_luminance(pyr3_renderer* r, const void* device_img, uint64_t pixels,
                                 int32_t kind, double* mean) {
  if (!r || !mean) return fail(PYR3_E_INVALID, "null argument");
  if (kind != PYR3_OUT_RGBA8 && kind != PYR3_OUT_RGBA32F && kind != PYR3_OUT_RGBA16F)
    return fail(PYR3_E_INVALID, "mean luminance: the image must be rgba8, rgba32f or rgba16f");
  if (pixels && (!device_img || (uintptr_t)device_img % 16))
    return fail(PYR3_E_INVALID, "the image must be a 16-byte aligned device buffer");
  cudaSetDevice(r->device);
  return luma_mean(r, device_img, pixels, kind, mean);
}

PYR3_API int pyr3_convert_display(const void* device_rgba32f, uint64_t pixels, int32_t out_kind,
                                  void* device_out, void* stream) {
  if (pyr3::out_bytes_per_pixel(out_kind) == 0) return fail(PYR3_E_INVALID, "unknown output kind");
  if (pixels == 0) return PYR3_OK;
  if (!device_rgba32f || !device_out || (uintptr_t)device_rgba32f % 16 || (uintptr_t)device_out % 16)
    return fail(PYR3_E_INVALID, "convert_display: images must be 16-byte aligned device buffers");
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(pyr3::launch_convert_display((const float*)device_rgba32f, pixels, out_kind, device_out,
                                        device_sms(dev), (cudaStream_t)stream));
  return PYR3_OK;
}

PYR3_API int pyr3_auto_exposure(pyr3_renderer* r, const pyr3_present_opts* p, uint64_t total_samples,
                                double target_mean, void* device_out, int32_t out_kind,
                                pyr3_brightness_fit* fit) {
  if (!r || !p || !device_out || !fit) return fail(PYR3_E_INVALID, "null argument");
  if ((uintptr_t)device_out % 16) return fail(PYR3_E_INVALID, "device_out must be 16-byte aligned");
  if (out_kind != PYR3_OUT_RGBA8 && out_kind != PYR3_OUT_RGBA32F && out_kind != PYR3_OUT_RGBA16F)
    return fail(PYR3_E_INVALID, "auto-exposure measures rgba8, rgba32f or rgba16f images");
  cudaSetDevice(r->device);
  const uint64_t pixels = (uint64_t)r->W * r->H;
  int rc = run_present(r, p, total_samples, device_out, out_kind, p->brightness);
  if (rc) return rc;
  double initial = 0.0;
  rc = luma_mean(r, device_out, pixels, out_kind, &initial);
  if (rc) return rc;
  return fit_brightness(p->brightness, target_mean, initial,
                        [&](double b, double* mean) -> int {
                          const int e = run_present(r, p, total_samples, device_out, out_kind, b);
                          return e ? e : luma_mean(r, device_out, pixels, out_kind, mean);
                        },
                        fit);
}

namespace {
// The queue and wave chaos kernels set sched[1] if one of their bounded
// waits ran out (a walker-queue wait, or a chunk copy that did not land) or
// a chunk copy was refused for a misaligned source, and the TMA-staged
// density and tonemap passes set bits 3 and 4 if a tile's copy did not
// land; it stays set until the next reset.
int check_sched(pyr3_renderer* r) {
  uint64_t f = 0;
  CUDA_TRY(cudaMemcpyAsync(&f, r->d_sched + 1, 8, cudaMemcpyDeviceToHost, r->stream));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  if (f & 24u) return fail(PYR3_E_CUDA, "present: a density or tonemap tile copy did not land within its bounded wait");
  if (f) return fail(PYR3_E_CUDA, "chaos kernel: a bounded wait (walker queue or chunk copy) exceeded its limit, or a chunk copy was refused");
  return PYR3_OK;
}
}  // namespace

PYR3_API int pyr3_read_histogram(pyr3_renderer* r, uint32_t* host_out) {
  if (!r || !host_out) return fail(PYR3_E_INVALID, "null argument");
  cudaSetDevice(r->device);
  CUDA_TRY(cudaMemcpyAsync(host_out, r->d_hist, (size_t)r->SW * r->SH * 16, cudaMemcpyDeviceToHost,
                           r->stream));
  return check_sched(r);
}

PYR3_API int pyr3_read_linear(pyr3_renderer* r, double k1, double k2, float* host_out) {
  if (!r || !host_out) return fail(PYR3_E_INVALID, "null argument");
  cudaSetDevice(r->device);
  const size_t bytes = (size_t)r->W * r->H * 16;
  int rc = ensure_out(r, bytes);
  if (rc) return rc;
  CUDA_TRY(pyr3::launch_linear_export(r->d_hist, r->W, r->H, r->os, k1, k2, (float*)r->d_out,
                                      r->stream));
  CUDA_TRY(cudaMemcpyAsync(host_out, r->d_out, bytes, cudaMemcpyDeviceToHost, r->stream));
  return check_sched(r);
}

PYR3_API int pyr3_read_index_map(pyr3_renderer* r, uint32_t* host_out) {
  if (!r || !host_out) return fail(PYR3_E_INVALID, "null argument");
  cudaSetDevice(r->device);
  CUDA_TRY(cudaMemcpyAsync(host_out, r->d_idx, (size_t)r->SW * r->SH * 4, cudaMemcpyDeviceToHost,
                           r->stream));
  CUDA_TRY(cudaStreamSynchronize(r->stream));
  return PYR3_OK;
}

PYR3_API int pyr3_sync(pyr3_renderer* r) {
  if (!r) return fail(PYR3_E_INVALID, "null renderer");
  cudaSetDevice(r->device);
  return check_sched(r);
}

PYR3_API int pyr3_info(pyr3_renderer* r, uint32_t* super_w, uint32_t* super_h, void** device_hist) {
  if (!r) return fail(PYR3_E_INVALID, "null renderer");
  if (super_w) *super_w = r->SW;
  if (super_h) *super_h = r->SH;
  if (device_hist) *device_hist = r->d_hist;
  return PYR3_OK;
}

PYR3_API int pyr3_counters(pyr3_renderer* r, uint64_t* samples, uint64_t* splats) {
  if (!r) return fail(PYR3_E_INVALID, "null renderer");
  uint64_t c[2] = {0, 0};
  cudaSetDevice(r->device);
  CUDA_TRY(cudaMemcpyAsync(c, r->d_counters, 16, cudaMemcpyDeviceToHost, r->stream));
  int rc = check_sched(r);
  if (rc) return rc;
  if (samples) *samples = c[0];
  if (splats) *splats = c[1];
  return PYR3_OK;
}

// ------------------------------------------------------ stage entry points
namespace {
// A throw-away genome shape of n linear xforms, for the pick / splat /
// seed stage kernels that live in the chaos module.
int stage_module(int n, std::shared_ptr<pyr3::ChaosModule>* m) {
  std::vector<float> xf((size_t)n * 116, 0.0f);
  for (int k = 0; k < n; ++k) {
    xf[(size_t)k * 116 + 7] = 1.0f;   // one variation
    xf[(size_t)k * 116 + 21] = 1.0f;  // linear, weight 1
  }
  pyr3::GenomeShape s;
  std::string e = pyr3::shape_from_packed(xf.data(), n, -1, &s);
  if (!e.empty()) return fail(PYR3_E_INVALID, e);
  std::string err;
  int rc = pyr3::get_chaos_module(s, kWpb, false, m, &err);
  if (rc) return fail(rc, err);
  return PYR3_OK;
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  ~DevBuf() { cudaFree(p); }
};
}  // namespace

PYR3_API int pyr3_seed_walkers(uint32_t seed, uint64_t base, uint32_t n, uint32_t* host_out) {
  if (!host_out || n == 0) return fail(PYR3_E_INVALID, "bad arguments");
  int rc = set_device(0);
  if (rc) return rc;
  std::shared_ptr<pyr3::ChaosModule> m;
  rc = stage_module(1, &m);
  if (rc) return rc;
  DevBuf<uint32_t> d;
  CUDA_TRY(cudaMalloc(&d.p, (size_t)n * 36 * 4));
  void* params[] = {&seed, &base, &n, &d.p};
  LAUNCH_TRY(m->seed_test, (n + kWpb - 1) / kWpb, kWpb, 0, nullptr, params);
  CUDA_TRY(cudaMemcpy(host_out, d.p, (size_t)n * 36 * 4, cudaMemcpyDeviceToHost));
  return PYR3_OK;
}

PYR3_API int pyr3_eval_variation(uint32_t idx, uint32_t n, const float* pts_xy, float weight,
                                 const float* params10, const float* a0, const float* a1,
                                 uint32_t* isaac, float* out_xy) {
  if (!pts_xy || !params10 || !a0 || !a1 || !isaac || !out_xy || n == 0)
    return fail(PYR3_E_INVALID, "bad arguments");
  int rc = set_device(0);
  if (rc) return rc;
  std::shared_ptr<pyr3::EvalModule> m;
  std::string err;
  rc = pyr3::get_eval_module((int)idx, &m, &err);
  if (rc) return fail(rc, err);
  DevBuf<float> dp, dprm, dout;
  DevBuf<uint32_t> dst;
  CUDA_TRY(cudaMalloc(&dp.p, (size_t)n * 8));
  CUDA_TRY(cudaMalloc(&dout.p, (size_t)n * 8));
  CUDA_TRY(cudaMalloc(&dprm.p, 40));
  CUDA_TRY(cudaMalloc(&dst.p, (size_t)n * 144));
  CUDA_TRY(cudaMemcpy(dp.p, pts_xy, (size_t)n * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dprm.p, params10, 40, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dst.p, isaac, (size_t)n * 144, cudaMemcpyHostToDevice));
  float4 A0 = make_float4(a0[0], a0[1], a0[2], a0[3]), A1 = make_float4(a1[0], a1[1], a1[2], a1[3]);
  void* params[] = {&n, &dp.p, &weight, &dprm.p, &A0, &A1, &dst.p, &dout.p};
  LAUNCH_TRY(m->eval, (n + 127) / 128, 128, 0, nullptr, params);
  CUDA_TRY(cudaMemcpy(out_xy, dout.p, (size_t)n * 8, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(isaac, dst.p, (size_t)n * 144, cudaMemcpyDeviceToHost));
  return PYR3_OK;
}

PYR3_API int pyr3_eval_dc_color(uint32_t idx, uint32_t n, const float* pts_xy, const float* v4,
                                const float* ve4, float* out_rgb, int32_t* hit) {
  if (!pts_xy || !v4 || !ve4 || !out_rgb || !hit || n == 0) return fail(PYR3_E_INVALID, "bad arguments");
  if (!pyr3::variation_is_dc((int)idx)) {
    for (uint32_t i = 0; i < n; ++i) hit[i] = 0;
    std::memset(out_rgb, 0, (size_t)n * 12);
    return PYR3_OK;
  }
  int rc = set_device(0);
  if (rc) return rc;
  std::shared_ptr<pyr3::EvalModule> m;
  std::string err;
  rc = pyr3::get_eval_module((int)idx, &m, &err);
  if (rc) return fail(rc, err);
  if (!m->dc) return fail(PYR3_E_UNSUPPORTED, "no direct colour kernel");
  const float prm[10] = {v4[2], v4[3], ve4[0], ve4[1], ve4[2], ve4[3], 0, 0, 0, 0};
  DevBuf<float> dp, dprm, dout;
  CUDA_TRY(cudaMalloc(&dp.p, (size_t)n * 8));
  CUDA_TRY(cudaMalloc(&dout.p, (size_t)n * 12));
  CUDA_TRY(cudaMalloc(&dprm.p, 40));
  CUDA_TRY(cudaMemcpy(dp.p, pts_xy, (size_t)n * 8, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dprm.p, prm, 40, cudaMemcpyHostToDevice));
  void* params[] = {&n, &dp.p, &dprm.p, &dout.p};
  LAUNCH_TRY(m->dc, (n + 127) / 128, 128, 0, nullptr, params);
  CUDA_TRY(cudaMemcpy(out_rgb, dout.p, (size_t)n * 12, cudaMemcpyDeviceToHost));
  for (uint32_t i = 0; i < n; ++i) hit[i] = 1;
  return PYR3_OK;
}

PYR3_API int pyr3_pick_stream(uint32_t n_xforms, const float* weights, const float* xaos,
                              uint32_t count, const int32_t* prev, const uint32_t* draws,
                              uint32_t* out) {
  if (!weights || !prev || !draws || !out || n_xforms == 0 || n_xforms > PYR3_MAX_XFORMS || count == 0)
    return fail(PYR3_E_INVALID, "bad arguments");
  int rc = set_device(0);
  if (rc) return rc;
  std::vector<uint16_t> starts;
  std::string err;
  if (!build_pick_starts((int)n_xforms, weights, xaos, &starts, &err)) return fail(PYR3_E_INVALID, err);
  std::shared_ptr<pyr3::ChaosModule> m;
  rc = stage_module((int)n_xforms, &m);
  if (rc) return rc;
  DevBuf<uint16_t> dst;
  DevBuf<int32_t> dprev;
  DevBuf<uint32_t> ddraw, dout;
  CUDA_TRY(cudaMalloc(&dst.p, starts.size() * 2));
  CUDA_TRY(cudaMalloc(&dprev.p, (size_t)count * 4));
  CUDA_TRY(cudaMalloc(&ddraw.p, (size_t)count * 4));
  CUDA_TRY(cudaMalloc(&dout.p, (size_t)count * 4));
  CUDA_TRY(cudaMemcpy(dst.p, starts.data(), starts.size() * 2, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dprev.p, prev, (size_t)count * 4, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(ddraw.p, draws, (size_t)count * 4, cudaMemcpyHostToDevice));
  void* params[] = {&dst.p, &count, &dprev.p, &ddraw.p, &dout.p};
  LAUNCH_TRY(m->pick_test, (count + 255) / 256, 256, 0, nullptr, params);
  CUDA_TRY(cudaMemcpy(out, dout.p, (size_t)count * 4, cudaMemcpyDeviceToHost));
  return PYR3_OK;
}

PYR3_API int pyr3_splat_points(uint32_t n, const float* pts, uint32_t width, uint32_t height,
                               float scale, float cx, float cy, float rotation_rad,
                               uint32_t palette_mode, const float* palette, int32_t aggregate,
                               uint32_t* hist_inout) {
  if (!pts || !palette || !hist_inout || n == 0 || width == 0 || height == 0)
    return fail(PYR3_E_INVALID, "bad arguments");
  int rc = set_device(0);
  if (rc) return rc;
  std::shared_ptr<pyr3::ChaosModule> m;
  {
    std::vector<float> xf(116, 0.0f);
    xf[7] = 1.0f;
    xf[21] = 1.0f;
    pyr3::GenomeShape s;
    pyr3::shape_from_packed(xf.data(), 1, -1, &s);
    std::string err;
    rc = pyr3::get_chaos_module(s, kWpb, aggregate != 0, &m, &err);
    if (rc) return fail(rc, err);
  }
  const size_t hb = (size_t)width * height * 16;
  DevBuf<float> dpts, dpal;
  DevBuf<uint32_t> dh;
  DevBuf<uint64_t> dcnt;
  CUDA_TRY(cudaMalloc(&dpts.p, (size_t)n * 16));
  CUDA_TRY(cudaMalloc(&dpal.p, 4096));
  CUDA_TRY(cudaMalloc(&dh.p, hb));
  CUDA_TRY(cudaMalloc(&dcnt.p, 16));
  CUDA_TRY(cudaMemcpy(dpts.p, pts, (size_t)n * 16, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dpal.p, palette, 4096, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dh.p, hist_inout, hb, cudaMemcpyHostToDevice));
  ChaosArgs A;
  std::memset(&A, 0, sizeof A);
  A.hist = dh.p;
  A.palette = dpal.p;
  A.width = width;
  A.height = height;
  A.scale = scale;
  A.cx = cx;
  A.cy = cy;
  A.cos_r = std::cos(rotation_rad);
  A.sin_r = std::sin(rotation_rad);
  A.palette_mode = palette_mode;
  A.counters = dcnt.p;
  void* params[] = {&A, &n, &dpts.p};
  LAUNCH_TRY(m->splat_test, (n + kWpb - 1) / kWpb, kWpb, 0, nullptr, params);
  CUDA_TRY(cudaMemcpy(hist_inout, dh.p, hb, cudaMemcpyDeviceToHost));
  return PYR3_OK;
}

PYR3_API int pyr3_density_tonemap(const uint32_t* hist, uint32_t width, uint32_t height,
                                  uint32_t oversample, float filter_radius,
                                  const pyr3_present_opts* p, uint64_t total_samples,
                                  float* out_rgba, float* filtered_out) {
  if (!hist || !p || !out_rgba || oversample == 0 || width == 0 || height == 0)
    return fail(PYR3_E_INVALID, "bad arguments");
  pyr3_opts o{width, height, oversample, filter_radius, 0};
  pyr3_renderer* r = nullptr;
  int rc = pyr3_create(&o, &r);
  if (rc) return rc;
  std::unique_ptr<pyr3_renderer, int (*)(pyr3_renderer*)> guard(r, pyr3_destroy);
  CUDA_TRY(cudaMemcpyAsync(r->d_hist, hist, (size_t)r->SW * r->SH * 16, cudaMemcpyHostToDevice, r->stream));
  rc = pyr3_present(r, p, total_samples, out_rgba, PYR3_OUT_RGBA32F);
  if (rc) return rc;
  if (filtered_out && p->density_on)
    CUDA_TRY(cudaMemcpy(filtered_out, r->d_filtered, (size_t)r->SW * r->SH * 16, cudaMemcpyDeviceToHost));
  return PYR3_OK;
}

// ------------------------------------------------ allocation-free present
// Density estimation + tonemap of a histogram the caller already holds on
// the device, into an image on the device, for callers that cannot
// allocate device memory (see noalloc.cu).  Same kernels and parameters as
// pyr3_present; the renderer-owned buffers are replaced by the library's
// fixed scratch array.
PYR3_API int pyr3_density_tonemap_noalloc(const uint32_t* device_hist, uint32_t width,
                                          uint32_t height, uint32_t oversample,
                                          float filter_radius, const pyr3_present_opts* p,
                                          uint64_t total_samples, void* device_out,
                                          int32_t out_kind, void* stream) {
  if (!device_hist || !p || !device_out || oversample == 0 || width == 0 || height == 0)
    return fail(PYR3_E_INVALID, "bad arguments");
  if (pyr3::out_bytes_per_pixel(out_kind) == 0) return fail(PYR3_E_INVALID, "unknown output kind");
  if (total_samples == 0) return fail(PYR3_E_INVALID, "total_samples must be positive");
  const uint64_t sw = (uint64_t)width * oversample, sh = (uint64_t)height * oversample;
  if (sw * sh > pyr3::kNoAllocMaxSuperPixels)
    return fail(PYR3_E_INVALID,
                "canvas too large for the allocation-free present: width*height*oversample^2 = " +
                    std::to_string(sw * sh) + " exceeds its fixed scratch of " +
                    std::to_string(pyr3::kNoAllocMaxSuperPixels) + " super-sampled pixels");
  cudaStream_t s = (cudaStream_t)stream;
  static float knorm[257];
  static std::once_flag knorm_once;
  std::call_once(knorm_once, [] { kernel_norm_lut(knorm); });
  pyr3::NoAllocScratch sc;
  CUDA_TRY(pyr3::noalloc_scratch(knorm, s, &sc));
  float taps[pyr3::kMaxTaps];
  const int fwidth = spatial_kernel(filter_radius > 0 ? filter_radius : 0.5f, (int)oversample, taps);
  const bool curves_on = p->curves && (p->curves_active & 31u);
  CUDA_TRY(pyr3::noalloc_write_tables(sc, taps, fwidth, curves_on ? p->curves : nullptr, s));
  // src/calibration.ts:37-43 in double, uploaded as f32.
  const double os2 = (double)oversample * (double)oversample;
  const float k1 = (float)((p->brightness * 255.0 * 268.0) / 256.0);
  const float k2 = (float)((os2 * p->scale * p->scale) / (255.0 * (double)total_samples));
  const float* filtered = nullptr;
  if (p->density_on) {
    pyr3::DeParams d;
    d.width = (uint32_t)sw;
    d.height = (uint32_t)sh;
    d.max_rad = (float)((double)p->de_max_rad * oversample + 1.0);
    d.min_rad = (float)((double)p->de_min_rad * oversample + 1.0);
    d.curve = p->de_curve;
    d.k1 = k1;
    d.k2 = k2;
    d.R = (int)std::ceil(std::min(std::max(d.max_rad, 0.0f), 256.0f));
    CUDA_TRY(pyr3::launch_density(device_hist, sc.filtered, d, sc.knorm, sc.kwtab, nullptr, s));
    filtered = sc.filtered;
  }
  pyr3::TonemapParams t;
  t.width = width;
  t.height = height;
  t.oversample = oversample;
  t.fwidth = (uint32_t)fwidth;
  t.k1 = k1;
  t.k2 = k2;
  t.gamma = p->gamma;
  t.vibrancy = p->vibrancy;
  t.highpow = p->highpow;
  t.linrange = p->linrange;
  t.bg[0] = p->background[0];
  t.bg[1] = p->background[1];
  t.bg[2] = p->background[2];
  t.transparent = p->transparent;
  t.curves_active = curves_on ? (p->curves_active & 31u) : 0u;
  t.hsl_active = p->hsl_active ? 1u : 0u;
  t.hsl_hue = p->hsl_hue;
  t.hsl_sat = p->hsl_sat;
  t.hsl_light = p->hsl_light;
  CUDA_TRY(pyr3::launch_tonemap(filtered ? nullptr : device_hist, filtered, t, sc.kern, sc.curves,
                                device_out, out_kind, nullptr, s));
  return PYR3_OK;
}

// ------------------------------------------------------------ build checks
PYR3_API int pyr3_jit_compile(const pyr3_genome* g, int32_t aggregate, uint64_t* cubin_bytes) {
  if (!g || !g->xforms) return fail(PYR3_E_INVALID, "null genome");
  pyr3::GenomeShape shape;
  std::string e = pyr3::shape_from_packed(g->xforms, (int)g->n_xforms, g->final_slot, &shape);
  if (!e.empty())
    return fail(e.find("not implemented") != std::string::npos ? PYR3_E_UNSUPPORTED : PYR3_E_INVALID, e);
  size_t n = 0;
  std::string err;
  int rc = pyr3::compile_chaos_only(shape, kWpb, aggregate != 0, &n, &err);
  if (rc) return fail(rc, err);
  if (cubin_bytes) *cubin_bytes = n;
  return PYR3_OK;
}

PYR3_API int pyr3_jit_source(const pyr3_genome* g, char* buf, uint64_t cap, uint64_t* len) {
  if (!g || !g->xforms) return fail(PYR3_E_INVALID, "null genome");
  pyr3::GenomeShape shape;
  std::string e = pyr3::shape_from_packed(g->xforms, (int)g->n_xforms, g->final_slot, &shape);
  if (!e.empty()) return fail(PYR3_E_INVALID, e);
  std::string src = pyr3::chaos_source(shape, kWpb, false);
  if (len) *len = src.size();
  if (buf && cap) {
    size_t n = std::min<size_t>(cap - 1, src.size());
    std::memcpy(buf, src.data(), n);
    buf[n] = 0;
  }
  return PYR3_OK;
}

PYR3_API int pyr3_jit_compile_variation(uint32_t idx, uint64_t* cubin_bytes) {
  size_t n = 0;
  std::string err;
  int rc = pyr3::compile_eval_only((int)idx, &n, &err);
  if (rc) return fail(rc, err);
  if (cubin_bytes) *cubin_bytes = n;
  return PYR3_OK;
}

PYR3_API int pyr3_variation_info(uint32_t idx, int32_t* implemented, int32_t* is_dc,
                                 const char** name) {
  if (idx >= (uint32_t)pyr3::kNumVariations) return fail(PYR3_E_INVALID, "index out of range");
  if (implemented) *implemented = pyr3::variation_implemented((int)idx) ? 1 : 0;
  if (is_dc) *is_dc = pyr3::variation_is_dc((int)idx) ? 1 : 0;
  if (name) *name = pyr3::variation_name((int)idx);
  return PYR3_OK;
}

PYR3_API int pyr3_pick_table(uint32_t n_xforms, const float* weights, const float* xaos,
                             uint32_t* table_out) {
  if (!weights || !table_out || n_xforms == 0 || n_xforms > PYR3_MAX_XFORMS)
    return fail(PYR3_E_INVALID, "bad arguments");
  std::vector<uint16_t> starts;
  std::string err;
  const int n = (int)n_xforms;
  if (!build_pick_starts(n, weights, xaos, &starts, &err)) return fail(PYR3_E_INVALID, err);
  for (int r = 0; r <= n; ++r) {
    const uint16_t* st = starts.data() + (size_t)r * n;
    for (uint32_t g = 0; g < kGrain; ++g) {
      uint32_t v = 0;
      for (int j = 1; j < n; ++j) v += g >= st[j] ? 1u : 0u;
      table_out[(size_t)r * kGrain + g] = v;
    }
  }
  return PYR3_OK;
}

// ------------------------------------------------------------------ timing
PYR3_API int pyr3_mark(pyr3_renderer* r, int32_t slot) {
  if (!r || slot < 0 || slot >= 8) return fail(PYR3_E_INVALID, "bad timing slot");
  cudaSetDevice(r->device);
  if (!r->marks[slot]) CUDA_TRY(cudaEventCreate(&r->marks[slot]));
  CUDA_TRY(cudaEventRecord(r->marks[slot], r->stream));
  return PYR3_OK;
}

PYR3_API int pyr3_elapsed(pyr3_renderer* r, int32_t a, int32_t b, float* ms) {
  if (!r || !ms || a < 0 || a >= 8 || b < 0 || b >= 8 || !r->marks[a] || !r->marks[b])
    return fail(PYR3_E_INVALID, "bad timing slots");
  cudaSetDevice(r->device);
  CUDA_TRY(cudaEventSynchronize(r->marks[b]));
  CUDA_TRY(cudaEventElapsedTime(ms, r->marks[a], r->marks[b]));
  return PYR3_OK;
}

PYR3_API int pyr3_splat_rate(pyr3_renderer* r, uint64_t splats, float* ms) {
  if (!r || !ms || splats == 0) return fail(PYR3_E_INVALID, "bad arguments");
  cudaSetDevice(r->device);
  CUDA_TRY(cudaEventRecord(r->ev0, r->stream));
  CUDA_TRY(pyr3::launch_splat_rate(r->d_hist, (uint64_t)r->SW * r->SH, splats, device_sms(r->device), r->stream));
  CUDA_TRY(cudaEventRecord(r->ev1, r->stream));
  CUDA_TRY(cudaEventSynchronize(r->ev1));
  CUDA_TRY(cudaEventElapsedTime(ms, r->ev0, r->ev1));
  return PYR3_OK;
}

PYR3_API int pyr3_flush_l2(pyr3_renderer* r, uint64_t bytes) {
  if (!r) return fail(PYR3_E_INVALID, "null renderer");
  cudaSetDevice(r->device);
  if (r->flush_bytes < bytes) {
    CUDA_TRY(cudaStreamSynchronize(r->stream));
    cudaFree(r->d_flush);
    r->d_flush = nullptr;
    CUDA_TRY(cudaMalloc(&r->d_flush, bytes));
    r->flush_bytes = bytes;
  }
  CUDA_TRY(cudaMemsetAsync(r->d_flush, 0x5a, bytes, r->stream));
  return PYR3_OK;
}
