// NVRTC specialisation of the chaos kernel per genome structure.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <atomic>
#include <memory>
#include <string>
#include <vector>

namespace pyr3 {

constexpr int kXformFloats = 116;
constexpr int kMaxVars = 8;
constexpr int kNumVariations = 326;
// Queue chaos kernel (genomes of up to kQueueMaxXforms xforms): one CTA of
// kQueueWarps warps per SM owning kQueueSlots walkers, whose records
// (kWalkerRecordBytes each) live in global memory; each warp stages
// kQueueStageWords u32 in shared memory, next to one ring per xform.
constexpr int kQueueMaxXforms = 32;
constexpr int kQueueWarps = 16;
constexpr int kQueueSlots = 2048;
constexpr int kQueueStageWords = 44 * 33 + 32;
constexpr int kWalkerRecordBytes = 192;
bool use_queue(int nxf);
// Wave chaos kernel (genomes of up to kWaveMaxXforms xforms): every walker
// of a launch resident in global memory as kWaveFields u32 per walker,
// grouped by next xform; one launch per iteration, kWaveBlock walkers per
// block.
constexpr int kWaveMaxXforms = 32;
constexpr int kWaveBlock = 256;
constexpr int kWaveFields = 49;
constexpr int kWaveMinBlocks = 3;
bool use_wave(int nxf);

// The part of a genome that changes the generated code: how many xforms,
// which variations each one sums (in slot order), which have a post
// affine, and the final xform.  Everything numeric is a runtime constant.
struct XformShape {
  std::vector<int> vars;  // variation index per active slot (97 = pre_blur)
  bool has_post = false;
};
struct GenomeShape {
  std::vector<XformShape> xf;  // regular xforms
  bool has_final = false;
  XformShape fin;
  std::string key() const;
};

// Extract the shape from packed 116-float records.  Returns an empty string
// on success or an error message.
std::string shape_from_packed(const float* xforms, int n, int final_slot, GenomeShape* out);

// Loaded through the runtime's library-management API (cudaLibrary_t /
// cudaKernel_t), so the shared library needs no link-time libcuda.
struct ChaosModule {
  cudaLibrary_t mod = nullptr;
  cudaKernel_t chaos = nullptr;
  cudaKernel_t pick_test = nullptr;
  cudaKernel_t splat_test = nullptr;
  cudaKernel_t seed_test = nullptr;
  void* c_xf = nullptr;
  size_t c_xf_bytes = 0;
  int nxf = 0;
  int wpb = 256;
  size_t smem = 0;      // dynamic shared memory of chaos_kernel
  int blocks_per_sm = 1;
  // chaos_queue_kernel (genomes of <= kQueueMaxXforms xforms), else null.
  cudaKernel_t queue = nullptr;
  size_t queue_smem = 0;
  int queue_blocks_per_sm = 0;
  // chaos_wave_kernel (genomes of <= kWaveMaxXforms xforms), else null.
  cudaKernel_t wave = nullptr;
  size_t wave_smem = 0;
  int wave_blocks_per_sm = 0;
  // Kernel choice of the autotuner for this structure: -1 not measured
  // yet, 0 chaos_kernel, 1 chaos_queue_kernel, 2 chaos_wave_kernel.
  std::atomic<int> choice{-1};
  ~ChaosModule();
};

struct EvalModule {
  cudaLibrary_t mod = nullptr;
  cudaKernel_t eval = nullptr;
  cudaKernel_t dc = nullptr;
  ~EvalModule();
};

// Compile (or load from the in-process / on-disk cache) the chaos module.
// Returns 0 or a PYR3_E_* code with *err set.
// instance > 0 loads a separate copy of the module (its own __constant__
// xform bank), for batches holding several genomes of one structure.
int get_chaos_module(const GenomeShape& s, int wpb, bool aggregate,
                     std::shared_ptr<ChaosModule>* out, std::string* err, int instance = 0);
// Compile the chaos modules of these shapes (aggregate[i] per shape) on
// parallel host threads, one per distinct source, into the cubin cache
// that get_chaos_module reads; compile errors are left for
// get_chaos_module to report.  NVRTC runs on the host: a batch of many new
// structures compiles in the time of the slowest few.
void precompile_chaos(const std::vector<GenomeShape>& shapes, const std::vector<bool>& aggregate, int wpb);
// Generate and compile (no device needed) the chaos module source; returns
// the cubin size through *bytes.  Used by CPU-side build checks.
int compile_chaos_only(const GenomeShape& s, int wpb, bool aggregate, size_t* bytes,
                       std::string* err);
// Generated NVRTC source of the chaos module for a shape.
std::string chaos_source(const GenomeShape& s, int wpb, bool aggregate);
// Compile the evaluator for variation `idx` without loading it.
int compile_eval_only(int idx, size_t* bytes, std::string* err);
// Module with the variation evaluator for variation `idx`.
int get_eval_module(int idx, std::shared_ptr<EvalModule>* out, std::string* err);
// True if the variation library implements `idx`.
bool variation_implemented(int idx);
const char* variation_name(int idx);
bool variation_is_dc(int idx);
// True if the variation may draw from the walker's random stream.
bool variation_draws(int idx);

}  // namespace pyr3
