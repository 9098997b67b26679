// NVRTC specialisation of the chaos kernel per genome structure, with an
// in-process module cache (per structure) and an on-disk cubin cache keyed
// by a hash of the generated source.
#include "jit.h"

#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <sstream>
#include <thread>
#include <unordered_set>

#include "pyr3.h"

namespace pyr3 {
namespace {
#include "gen/jit_sources.inc"

std::mutex g_mu;
std::map<std::string, std::weak_ptr<ChaosModule>> g_chaos_cache;
// Cubins compiled or read by this process, by cache path: a compile on
// another thread (precompile_chaos) lands here even where the cache
// directory cannot be written.
std::mutex g_cubin_mu;
std::map<std::string, std::string> g_cubins;
std::map<int, std::shared_ptr<EvalModule>> g_eval_cache;

uint64_t fnv1a(const std::string& s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char ch : s) {
    h ^= ch;
    h *= 1099511628211ull;
  }
  return h;
}

// Cubin cache: $PYR3_CACHE_DIR; else a `_cubins` directory beside this
// shared library, if one exists (the build fills it, so a copy of the
// package carries its compiled modules); else ~/.cache/pyr3_b200.
std::string cache_dir() {
  const char* d = std::getenv("PYR3_CACHE_DIR");
  std::string dir;
  Dl_info info;
  struct stat st;
  if (d && *d) {
    dir = d;
  } else if (dladdr((void*)&cache_dir, &info) && info.dli_fname &&
             std::strrchr(info.dli_fname, '/') &&
             stat((std::string(info.dli_fname, std::strrchr(info.dli_fname, '/')) + "/_cubins").c_str(), &st) == 0 &&
             S_ISDIR(st.st_mode)) {
    dir = std::string(info.dli_fname, std::strrchr(info.dli_fname, '/')) + "/_cubins";
  } else {
    const char* home = std::getenv("HOME");
    dir = std::string(home && *home ? home : "/tmp") + "/.cache/pyr3_b200";
  }
  std::string acc;
  std::stringstream ss(dir);
  std::string part;
  if (!dir.empty() && dir[0] == '/') acc = "";
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    acc += "/" + part;
    mkdir(acc.c_str(), 0755);
  }
  return dir;
}

bool read_file(const std::string& path, std::string* out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  std::stringstream ss;
  ss << f.rdbuf();
  *out = ss.str();
  return !out->empty();
}

void write_file_atomic(const std::string& path, const std::string& data) {
  // Unique per process and thread: two threads may write the same module.
  std::string tmp = path + ".tmp." + std::to_string(getpid()) + "." +
                    std::to_string(std::hash<std::thread::id>()(std::this_thread::get_id()));
  {
    std::ofstream f(tmp, std::ios::binary);
    if (!f) return;
    f.write(data.data(), (std::streamsize)data.size());
  }
  std::rename(tmp.c_str(), path.c_str());
}

std::string library_source() {
  std::string s = kSrcCore;
  for (int i = 0; i < kNumVlib; ++i) {
    s += "\n";
    s += kSrcVlib[i];
  }
  return s;
}

// Compile `src` to a sm_100a cubin (disk-cached).
int compile_cubin(const std::string& src, const std::string& name, std::string* cubin,
                  std::string* err) {
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--fmad=true",
                        "-default-device"};
  const int nopts = 4;
  std::string key = src;
  for (int i = 0; i < nopts; ++i) key += opts[i];
  char hex[32];
  std::snprintf(hex, sizeof hex, "%016llx", (unsigned long long)fnv1a(key));
  const std::string path = cache_dir() + "/" + name + "-" + hex + ".cubin";
  {
    std::lock_guard<std::mutex> lk(g_cubin_mu);
    auto it = g_cubins.find(path);
    if (it != g_cubins.end()) {
      *cubin = it->second;
      return PYR3_OK;
    }
  }
  if (read_file(path, cubin)) {
    std::lock_guard<std::mutex> lk(g_cubin_mu);
    g_cubins[path] = *cubin;
    return PYR3_OK;
  }

  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src.c_str(), (name + ".cu").c_str(), 0, nullptr, nullptr) !=
      NVRTC_SUCCESS) {
    *err = "nvrtcCreateProgram failed";
    return PYR3_E_NVRTC;
  }
  nvrtcResult rc = nvrtcCompileProgram(prog, nopts, opts);
  size_t log_n = 0;
  nvrtcGetProgramLogSize(prog, &log_n);
  std::string log(log_n, '\0');
  if (log_n > 1) nvrtcGetProgramLog(prog, &log[0]);
  if (rc != NVRTC_SUCCESS) {
    *err = std::string("NVRTC compile of ") + name + " failed: " + nvrtcGetErrorString(rc) + "\n" +
           log.substr(0, 8000);
    nvrtcDestroyProgram(&prog);
    return PYR3_E_NVRTC;
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  cubin->assign(n, '\0');
  nvrtcGetCUBIN(prog, &(*cubin)[0]);
  nvrtcDestroyProgram(&prog);
  write_file_atomic(path, *cubin);
  std::lock_guard<std::mutex> lk(g_cubin_mu);
  g_cubins[path] = *cubin;
  return PYR3_OK;
}

const char* cu_err(cudaError_t r) { return cudaGetErrorString(r); }

// ---- code generation ----------------------------------------------------
// One xform chain, following apply_xform_chain (chaos.wgsl:8226-8267) and
// apply_pre_blur (chaos.wgsl:8164-8181): affine, pre_blur deltas (five
// draws each, in slot order), variation sum in slot order with the
// direct-colour check after each slot, post affine, colour contraction.
// The affines, the pre_blur offset, the variation sum and the colour mix
// round every product and sum on its own (aff_rn, mix_rn, __fadd_rn), as
// the reference's f32 expressions do, so no FMA contraction moves their
// last bit; pre_blur's cos / sin are the f32 roundings of the double
// values (sincos_rn).  An affine-only genome then iterates bit for bit as
// the reference does.
std::string gen_chain(const XformShape& x, const std::string& base, const char* pz) {
  std::ostringstream o;
  o << "  const float* X = " << base << ";\n";
  o << "  float2 t = f2(aff_rn(X[0], p.x, X[1], p.y, X[2]), aff_rn(X[4], p.x, X[5], p.y, X[6]));\n";
  for (size_t j = 0; j < x.vars.size(); ++j) {
    if (x.vars[j] != 97) continue;
    const int wi = 21 + 4 * (int)j;
    o << "  { const float g0 = rand01(c.rng), g1 = rand01(c.rng), g2 = rand01(c.rng), "
         "g3 = rand01(c.rng);\n"
      << "    const float g = __fmul_rn(X[" << wi
      << "], __fsub_rn(__fadd_rn(__fadd_rn(__fadd_rn(g0, g1), g2), g3), 2.0f));\n"
      << "    const float ang = __fmul_rn(rand01(c.rng), P_TAU);\n"
      << "    const float2 sc = sincos_rn(ang);\n"
      << "    t = f2(__fadd_rn(t.x, __fmul_rn(sc.y, g)), __fadd_rn(t.y, __fmul_rn(sc.x, g))); }\n";
  }
  o << "  float2 acc = f2(0.0f, 0.0f);\n";
  for (size_t j = 0; j < x.vars.size(); ++j) {
    const int v = x.vars[j];
    const int b = 20 + 4 * (int)j, e = 52 + 4 * (int)j, e2 = 84 + 4 * (int)j;
    const bool dc = variation_is_dc(v);
    const bool pos = v != 97 && !(v >= 99 && v <= 101);
    if (!pos && !dc) continue;
    o << "  { const float P" << j << "[10] = {X[" << b + 2 << "], X[" << b + 3 << "], X[" << e
      << "], X[" << e + 1 << "], X[" << e + 2 << "], X[" << e + 3 << "], X[" << e2 << "], X["
      << e2 + 1 << "], X[" << e2 + 2 << "], X[" << e2 + 3 << "]};\n";
    if (pos)
      o << "    { const float2 v = var_" << variation_name(v) << "(t, X[" << b + 1 << "], P" << j
        << ", c); acc = f2(__fadd_rn(acc.x, v.x), __fadd_rn(acc.y, v.y)); }\n";
    if (dc)
      o << "    if (X[11] > 0.5f && X[" << b + 1 << "] > 0.0f) { o.dc = dc_" << variation_name(v)
        << "(t, P" << j << "); o.dc_hit = 1; }\n";
    o << "  }\n";
  }
  if (x.has_post)
    o << "  acc = f2(aff_rn(X[12], acc.x, X[13], acc.y, X[14]), aff_rn(X[16], acc.x, X[17], acc.y, "
         "X[18]));\n";
  o << "  o.pv = acc;\n  o.nz = mix_rn(" << pz << ", X[8], X[9]);\n";
  return o.str();
}

}  // namespace

bool use_queue(int nxf) { return nxf >= 1 && nxf <= kQueueMaxXforms; }
bool use_wave(int nxf) { return nxf >= 1 && nxf <= kWaveMaxXforms; }

namespace {

std::string gen_chaos_source(const GenomeShape& s, int wpb, bool aggregate) {
  const int nxf = (int)s.xf.size();
  std::ostringstream o;
  // A final xform whose variations draw nothing may be skipped while a
  // walker burns in (its result is not splatted then); with an opacity gate
  // below 1 it still runs, since the gate draws.
  bool final_rng_free = s.has_final;
  for (int v : s.fin.vars) final_rng_free = final_rng_free && !variation_draws(v);
  o << "#define NXF " << nxf << "\n#define WPB " << wpb << "\n#define HAS_FINAL "
    << (s.has_final ? 1 : 0) << "\n#define FINAL_RNG_FREE " << (final_rng_free ? 1 : 0)
    << "\n#define FINAL_SLOT " << nxf << "\n#define PICK_LINEAR "
    << (nxf <= 16 ? 1 : 0) << "\n#define AGGREGATE " << (aggregate ? 1 : 0) << "\n#define QUEUE "
    << (use_queue(nxf) ? 1 : 0) << "\n#define QWARPS " << kQueueWarps << "\n#define WAVE "
    << (use_wave(nxf) ? 1 : 0) << "\n#define WAVE_MINB " << kWaveMinBlocks << "\n";
  o << library_source() << "\n";
  o << kSrcChaosPre << "\n";
  o << "VDEV void xform_chain(int k, float2 p, float pz, Ctx& c, ChainOut& o) {\n  switch (k) {\n";
  for (int k = 0; k < nxf; ++k) {
    o << "  case " << k << ": {\n"
      << gen_chain(s.xf[k], "c_xf + " + std::to_string(k * kXformFloats), "pz") << "  } break;\n";
  }
  o << "  default: o.pv = p; o.nz = pz; break;\n  }\n}\n";
  o << "VDEV void final_chain(float2 p, float nz, Ctx& c, ChainOut& o) {\n";
  if (s.has_final) o << gen_chain(s.fin, "c_xf + " + std::to_string(nxf * kXformFloats), "nz");
  o << "}\n";
  o << kSrcChaosKernel << "\n";
  return o.str();
}

}  // namespace

ChaosModule::~ChaosModule() {
  if (mod) cudaLibraryUnload(mod);
}
EvalModule::~EvalModule() {
  if (mod) cudaLibraryUnload(mod);
}

bool variation_implemented(int idx) {
  return idx >= 0 && idx < kNumVariations && kVarImpl[idx] != 0;
}
const char* variation_name(int idx) {
  return idx >= 0 && idx < kNumVariations ? kVarNames[idx] : "?";
}
bool variation_is_dc(int idx) { return idx >= 0 && idx < kNumVariations && kVarDc[idx] != 0; }
// True if the variation may draw from the walker's random stream (pre_blur,
// index 97, always draws; a scan of the library's sources marks the rest).
bool variation_draws(int idx) { return idx == 97 || (idx >= 0 && idx < kNumVariations && kVarRng[idx] != 0); }

std::string GenomeShape::key() const {
  std::ostringstream o;
  for (const auto& x : xf) {
    o << (x.has_post ? 'P' : 'x');
    for (int v : x.vars) o << v << ',';
    o << ';';
  }
  if (has_final) {
    o << "F" << (fin.has_post ? 'P' : 'x');
    for (int v : fin.vars) o << v << ',';
  }
  return o.str();
}

static std::string shape_one(const float* X, XformShape* s) {
  float nv = X[7];
  if (!(nv >= 0.0f) || !std::isfinite(nv)) return "xform has an invalid variation count";
  int n = (int)nv;
  if (n > kMaxVars) n = kMaxVars;  // min(u32(a1.w), MAX_VARS_PER_XFORM)
  s->vars.clear();
  for (int j = 0; j < n; ++j) {
    float fi = X[20 + 4 * j];
    if (!(fi >= 0.0f) || !std::isfinite(fi)) return "variation index is not a non-negative number";
    int idx = (int)fi;
    if (idx == 97 || variation_implemented(idx) || variation_is_dc(idx)) {
      s->vars.push_back(idx);
    } else if (idx >= kNumVariations) {
      s->vars.push_back(-1);  // the reference's default case contributes (0, 0)
    } else {
      return std::string("variation ") + std::to_string(idx) + " (" + variation_name(idx) +
             ") is not implemented in this library";
    }
  }
  // Out-of-range indices contribute nothing: drop them from the generated code.
  std::vector<int> kept;
  for (int v : s->vars)
    if (v >= 0) kept.push_back(v);
  s->vars.swap(kept);
  s->has_post = X[15] != 0.0f;
  return "";
}

std::string shape_from_packed(const float* xforms, int n, int final_slot, GenomeShape* out) {
  if (n < 1 || n > PYR3_MAX_XFORMS) return "n_xforms must be in 1..128";
  if (final_slot != -1 && final_slot != n) return "final_slot must be -1 or n_xforms";
  out->xf.assign(n, XformShape());
  for (int k = 0; k < n; ++k) {
    std::string e = shape_one(xforms + (size_t)k * kXformFloats, &out->xf[k]);
    if (!e.empty()) return "xform " + std::to_string(k) + ": " + e;
  }
  out->has_final = final_slot >= 0;
  if (out->has_final) {
    std::string e = shape_one(xforms + (size_t)n * kXformFloats, &out->fin);
    if (!e.empty()) return "final xform: " + e;
  }
  return "";
}

void precompile_chaos(const std::vector<GenomeShape>& shapes, const std::vector<bool>& aggregate, int wpb) {
  std::unordered_set<std::string> seen;
  std::vector<const std::string*> srcs;
  for (size_t i = 0; i < shapes.size(); ++i) {
    auto ins = seen.insert(gen_chaos_source(shapes[i], wpb, aggregate[i]));
    if (ins.second) srcs.push_back(&*ins.first);
  }
  if (srcs.size() < 2) return;  // nothing to overlap
  const size_t nt = std::min<size_t>(srcs.size(), std::max(1u, std::thread::hardware_concurrency()));
  std::atomic<size_t> next{0};
  std::vector<std::thread> ts;
  for (size_t t = 0; t < nt; ++t)
    ts.emplace_back([&] {
      for (size_t i; (i = next++) < srcs.size();) {
        std::string cubin, err;
        compile_cubin(*srcs[i], "chaos", &cubin, &err);  // errors surface in get_chaos_module
      }
    });
  for (auto& t : ts) t.join();
}

int get_chaos_module(const GenomeShape& s, int wpb, bool aggregate,
                     std::shared_ptr<ChaosModule>* out, std::string* err, int instance) {
  const std::string key = s.key() + "|w" + std::to_string(wpb) + (aggregate ? "|A" : "") +
                          (instance > 0 ? "|i" + std::to_string(instance) : "");
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_chaos_cache.find(key);
    if (it != g_chaos_cache.end()) {
      if (auto sp = it->second.lock()) {
        *out = sp;
        return PYR3_OK;
      }
    }
  }
  const std::string src = gen_chaos_source(s, wpb, aggregate);
  std::string cubin;
  int rc = compile_cubin(src, "chaos", &cubin, err);
  if (rc) return rc;
  auto m = std::make_shared<ChaosModule>();
  cudaError_t cr = cudaLibraryLoadData(&m->mod, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
  if (cr != cudaSuccess) {
    *err = std::string("cudaLibraryLoadData: ") + cu_err(cr);
    return PYR3_E_CUDA;
  }
  if (cudaLibraryGetKernel(&m->chaos, m->mod, "chaos_kernel") != cudaSuccess ||
      cudaLibraryGetKernel(&m->pick_test, m->mod, "pick_test_kernel") != cudaSuccess ||
      cudaLibraryGetKernel(&m->splat_test, m->mod, "splat_test_kernel") != cudaSuccess ||
      cudaLibraryGetKernel(&m->seed_test, m->mod, "seed_test_kernel") != cudaSuccess ||
      cudaLibraryGetGlobal(&m->c_xf, &m->c_xf_bytes, m->mod, "c_xf") != cudaSuccess) {
    *err = "chaos module is missing a kernel or c_xf";
    return PYR3_E_CUDA;
  }
  const int nxf = (int)s.xf.size();
  m->nxf = nxf;
  m->wpb = wpb;
  const size_t pick_u16 = ((size_t)(nxf + 1) * nxf + 1) & ~(size_t)1;
  m->smem = (size_t)36 * wpb * 4 + 256 * 16 + (size_t)9 * wpb * 4 + (size_t)2 * wpb * 4 +
            (size_t)wpb * 2 + pick_u16 * 2 + (size_t)(nxf + 2) * 4;
  cudaFuncSetAttribute((const void*)m->chaos, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->smem);
  int nb = 0;
  cr = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)m->chaos, wpb, m->smem);
  if (cr != cudaSuccess || nb < 1) {
    *err = "chaos kernel cannot be resident (shared memory / registers)";
    return PYR3_E_CUDA;
  }
  if (use_queue(nxf)) {
    // Shared memory of the queue kernel (chaos_kernel.cuh, QUEUE): palette,
    // one staging area per warp, rings [NXF][QP] u16, pick boundaries,
    // heads, tails, live counter, current ring.
    if (cudaLibraryGetKernel(&m->queue, m->mod, "chaos_queue_kernel") != cudaSuccess) {
      *err = "chaos module is missing chaos_queue_kernel";
      return PYR3_E_CUDA;
    }
    m->queue_smem = 256 * 16 + (size_t)kQueueWarps * kQueueStageWords * 4 +
                    (size_t)nxf * kQueueSlots * 2 + pick_u16 * 2 + (size_t)nxf * 8 + 8;
    cudaFuncSetAttribute((const void*)m->queue, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)m->queue_smem);
    int qb = 0;
    cr = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&qb, (const void*)m->queue, kQueueWarps * 32,
                                                       m->queue_smem);
    if (cr == cudaSuccess && qb >= 1) m->queue_blocks_per_sm = qb;
    else m->queue = nullptr;  // not resident: the barrier kernel serves this structure
  }
  if (use_wave(nxf)) {
    // Shared memory of the wave kernel (chaos_kernel.cuh, WAVE): palette,
    // ISAAC state + stash [43][WB], walker fields [6][WB], sorted destinations,
    // per-xform counts / offsets / bases, work item, sorted walker ids and
    // keys, pick boundaries.
    if (cudaLibraryGetKernel(&m->wave, m->mod, "chaos_wave_kernel") != cudaSuccess) {
      *err = "chaos module is missing chaos_wave_kernel";
      return PYR3_E_CUDA;
    }
    const size_t wb = kWaveBlock;
    m->wave_smem = 256 * 16 + 43 * wb * 4 + 6 * wb * 4 + wb * 4 + (size_t)(3 * nxf + 1) * 4 + 3 * 4 +
                   wb * 2 + wb + (size_t)(nxf + 1) * nxf * 2;
    cudaFuncSetAttribute((const void*)m->wave, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)m->wave_smem);
    int wbn = 0;
    cr = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wbn, (const void*)m->wave, kWaveBlock,
                                                       m->wave_smem);
    if (cr == cudaSuccess && wbn >= 1) m->wave_blocks_per_sm = wbn;
    else m->wave = nullptr;  // not resident: another kernel serves this structure
  }
  m->blocks_per_sm = nb;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_chaos_cache[key] = m;
  }
  *out = m;
  return PYR3_OK;
}

std::string chaos_source(const GenomeShape& s, int wpb, bool aggregate) {
  return gen_chaos_source(s, wpb, aggregate);
}

int compile_chaos_only(const GenomeShape& s, int wpb, bool aggregate, size_t* bytes,
                       std::string* err) {
  std::string cubin;
  int rc = compile_cubin(gen_chaos_source(s, wpb, aggregate), "chaos", &cubin, err);
  if (rc == PYR3_OK && bytes) *bytes = cubin.size();
  return rc;
}

static std::string eval_source(int idx) {
  std::ostringstream o;
  o << library_source() << "\n";
  o << "#define EVAL_VAR var_" << variation_name(idx) << "\n";
  if (variation_is_dc(idx)) o << "#define EVAL_DC dc_" << variation_name(idx) << "\n";
  o << kSrcEval << "\n";
  return o.str();
}

int compile_eval_only(int idx, size_t* bytes, std::string* err) {
  if (!variation_implemented(idx)) {
    *err = "not implemented";
    return PYR3_E_UNSUPPORTED;
  }
  std::string cubin;
  int rc = compile_cubin(eval_source(idx), std::string("eval_") + variation_name(idx), &cubin, err);
  if (rc == PYR3_OK && bytes) *bytes = cubin.size();
  return rc;
}

int get_eval_module(int idx, std::shared_ptr<EvalModule>* out, std::string* err) {
  if (!variation_implemented(idx)) {
    *err = std::string("variation ") + std::to_string(idx) + " not implemented";
    return PYR3_E_UNSUPPORTED;
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_eval_cache.find(idx);
    if (it != g_eval_cache.end()) {
      *out = it->second;
      return PYR3_OK;
    }
  }
  std::string cubin;
  int rc = compile_cubin(eval_source(idx), std::string("eval_") + variation_name(idx), &cubin, err);
  if (rc) return rc;
  auto m = std::make_shared<EvalModule>();
  cudaError_t cr = cudaLibraryLoadData(&m->mod, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
  if (cr != cudaSuccess) {
    *err = std::string("cudaLibraryLoadData: ") + cu_err(cr);
    return PYR3_E_CUDA;
  }
  if (cudaLibraryGetKernel(&m->eval, m->mod, "eval_kernel") != cudaSuccess) {
    *err = "eval module is missing eval_kernel";
    return PYR3_E_CUDA;
  }
  if (cudaLibraryGetKernel(&m->dc, m->mod, "dc_kernel") != cudaSuccess) {
    m->dc = nullptr;
    cudaGetLastError();
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_eval_cache[idx] = m;
  }
  *out = m;
  return PYR3_OK;
}

}  // namespace pyr3
