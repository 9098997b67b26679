// Fixed scratch memory for the allocation-free present (noalloc.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace pyr3 {

// Density-estimation output capacity: super-sampled pixels (f32 x 4 each).
constexpr size_t kNoAllocMaxSuperPixels = (size_t)1 << 20;
extern const size_t kNoAllocScratchBytes;

// Device addresses inside the fixed array, for the current device.
struct NoAllocScratch {
  const float* knorm;  // 257-entry kernel-norm LUT
  const float* kwtab;  // density exp-weight table
  float* kern;         // spatial-filter taps (written per call)
  float* curves;       // colour-curves LUT, 5 x 256 f32 (written per call when used)
  float* filtered;     // density output, kNoAllocMaxSuperPixels x 4 f32
};

// Addresses of the array on the current device.  The first call on a
// device looks the array up with cudaGetSymbolAddress and fills the tables
// from knorm_host (on `stream`, then waits for it); later calls only
// return the addresses.
cudaError_t noalloc_scratch(const float* knorm_host, cudaStream_t stream, NoAllocScratch* out);

// Write one call's spatial-filter taps (n_taps <= kMaxTaps) and, when
// `curves` is not null, its 5 x 256 colour-curves LUT into the array, by a
// kernel on `stream` that receives the values as its parameter.
cudaError_t noalloc_write_tables(const NoAllocScratch& sc, const float* taps, int n_taps,
                                 const float* curves, cudaStream_t stream);

}  // namespace pyr3
