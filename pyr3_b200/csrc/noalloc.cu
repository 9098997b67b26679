// Scratch memory for the allocation-free present (pyr3_density_tonemap_noalloc).
//
// Some callers cannot allocate device memory: code running where the
// allocator is owned by someone else (a host application's memory pool or
// arena, a plugin inside another engine's frame loop), or code that must
// not allocate once it is running.  The present pass normally keeps its
// density-estimation output and lookup tables in buffers the renderer
// allocates; for those callers the same kernels run on the fixed array
// below instead, and the caller passes only its own input histogram and
// output image.
//
// The array is part of the library's device code: every GPU that loads it
// holds these kNoAllocScratchBytes (about 16.4 MiB) until the process
// exits.  It holds at most kNoAllocMaxSuperPixels super-sampled pixels of
// density-estimation output.  All calls on a device share it, so calls
// whose GPU work overlaps (different streams or host threads) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "noalloc.h"
#include "passes.h"

namespace pyr3 {
namespace {

constexpr size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Layout of the scratch array: kernel-norm LUT (257 f32), spatial-filter
// taps, colour-curves LUT (5 x 256 f32), the exp-weight table of the density
// pass, then the density output (f32 x 4 per super-sampled pixel).
constexpr size_t kKwRegionFloats = 90112;  // >= kw_table_floats() (checked at set-up)
constexpr size_t kOffKnorm = 0;
constexpr size_t kOffKern = kOffKnorm + align256(257 * sizeof(float));
constexpr size_t kOffCurves = kOffKern + align256(kMaxTaps * sizeof(float));
constexpr size_t kOffKw = kOffCurves + align256(5 * 256 * sizeof(float));
constexpr size_t kOffFiltered = kOffKw + align256(kKwRegionFloats * sizeof(float));
constexpr size_t kScratchBytes = kOffFiltered + kNoAllocMaxSuperPixels * 4 * sizeof(float);

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_base[kMaxDevices] = {};  // device address of the array, per device

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

const size_t kNoAllocScratchBytes = kScratchBytes;

// Once per device (the current one): look up the array's device address --
// in host code its name is only a host-side stand-in, not a device
// address -- then fill the tables, which later calls only read.  Nothing
// else in the array needs to start at zero: each call writes the taps, the
// curves LUT when it uses curves, and, when density estimation is on, every
// density-output pixel it later reads.
cudaError_t noalloc_scratch(const float* knorm_host, cudaStream_t stream, NoAllocScratch* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (kw_table_floats() > kKwRegionFloats) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_base[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    unsigned char* base = (unsigned char*)p;
    // The LUT goes up on `stream`, the same stream as the table built from
    // it, so the table never reads a half-written LUT whatever kind of
    // stream the caller passes.
    e = cudaMemcpyAsync(base + kOffKnorm, knorm_host, 257 * sizeof(float), cudaMemcpyHostToDevice,
                        stream);
    if (e != cudaSuccess) return e;
    e = build_kw_table((const float*)(base + kOffKnorm), (float*)(base + kOffKw), stream);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return e;
    g_base[dev] = base;
  }
  unsigned char* base = g_base[dev];
  out->knorm = (const float*)(base + kOffKnorm);
  out->kwtab = (const float*)(base + kOffKw);
  out->kern = (float*)(base + kOffKern);
  out->curves = (float*)(base + kOffCurves);
  out->filtered = (float*)(base + kOffFiltered);
  return cudaSuccess;
}

namespace {
// The per-call values, carried to the device as one kernel parameter: the
// launch copies them, so no host buffer has to outlive the call and no copy
// from pageable host memory is queued.
struct NoAllocCallTables {
  float taps[kMaxTaps];
  float curves[5 * 256];
  unsigned int n_taps;
  unsigned int has_curves;
};

__global__ void k_noalloc_tables(const __grid_constant__ NoAllocCallTables t, float* kern,
                                 float* curves) {
  const unsigned int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < t.n_taps) kern[i] = t.taps[i];
  if (t.has_curves && i < 5u * 256u) curves[i] = t.curves[i];
}
}  // namespace

cudaError_t noalloc_write_tables(const NoAllocScratch& sc, const float* taps, int n_taps,
                                 const float* curves, cudaStream_t stream) {
  if (n_taps < 1 || n_taps > kMaxTaps) return cudaErrorInvalidValue;
  NoAllocCallTables t;
  for (int i = 0; i < n_taps; ++i) t.taps[i] = taps[i];
  for (int i = n_taps; i < kMaxTaps; ++i) t.taps[i] = 0.0f;
  t.n_taps = (unsigned int)n_taps;
  t.has_curves = curves ? 1u : 0u;
  for (int i = 0; i < 5 * 256; ++i) t.curves[i] = curves ? curves[i] : 0.0f;
  k_noalloc_tables<<<5, 256, 0, stream>>>(t, sc.kern, sc.curves);
  return cudaGetLastError();
}

}  // namespace pyr3
