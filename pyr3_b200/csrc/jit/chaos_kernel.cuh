// pyr3-b200 persistent chaos-game kernel (NVRTC template).
//
// The host generator (csrc/jit.cpp) prepends, per genome STRUCTURE (xform
// count, each xform's variation list, post-affine flags, final xform):
//   #define NXF / WPB / HAS_FINAL / FINAL_SLOT / PICK_LINEAR / AGGREGATE
//   VDEV void xform_chain(int k, float2 p, float pz, Ctx& c, ChainOut& o);
//   VDEV void final_chain(float2 p, float pz, Ctx& c, ChainOut& o);
// and every numeric genome value (affines, weights, parameters, colours)
// is read from c_xf[] (the reference's 116-float packed xform records,
// src/genome.ts:293-313), so one compiled module serves every frame of an
// animation whose structure does not change.
//
// Per walker the loop follows chaos_main (src/shaders/chaos.wgsl:8269-8731):
// random start point, `fuse` burn-in iterations, xform pick from the
// (weight x xaos) table, affine -> pre_blur -> sum of variations -> post
// affine -> colour contraction, bad-value reseed with up to 4 retries, final
// xform lens with opacity gate, scale-relative jitter, and a saturating
// 4 x u32 splat.  RNG draws happen in exactly the reference's order.
//
// B200 organisation: one CTA = WPB walkers.  Each round is three phases
// separated by __syncthreads():
//   A  walker-owned: draw the pick, bucket the walker by xform (counting
//      sort in shared memory);
//   B  slot-owned: thread s runs the xform of the s-th walker in xform
//      order, so a warp executes one xform's straight-line code instead of
//      diverging over up to NXF of them;
//   C  walker-owned: bad-value retry logic, final xform, jitter, splat.
// ISAAC state for all WPB walkers lives in shared memory as [36][WPB] u32,
// so any thread can draw from any walker's stream conflict-free.
#pragma once

#ifndef MAXRANK
#define MAXRANK (NXF + 1)
#endif
#ifndef FINAL_RNG_FREE
#define FINAL_RNG_FREE 0
#endif

__constant__ float c_xf[(NXF + HAS_FINAL) * 116];

struct ChainOut {
  float2 pv;    // chain output after the post affine
  float nz;     // contracted colour coordinate
  float3 dc;    // direct-colour override
  int dc_hit;   // 1 if a DC variation coloured this point
};

struct ChaosArgs {
  u32* hist;               // superW x superH x 4 (R, G, B, count)
  u32* idx_sum;            // superW x superH (capture_index) or null
  const float* palette;    // 256 x RGBA f32
  const unsigned short* pick_start;  // (NXF+1) x NXF boundaries, see below
  u64 walker_base;         // global index of this launch's walker 0
  u64 n_walkers;           // walkers in this launch
  u64 iters_base;          // post-fuse iterations of every walker
  u64 iters_extra;         // walkers [0, iters_extra) run one more
  u32 fuse;
  u32 width, height;       // super-res canvas
  float scale, cx, cy;     // scale already multiplied by oversample
  float cos_r, sin_r;      // camera rotation
  u32 seed;
  float jitter;            // scale-relative walker jitter (default 1e-7)
  u32 palette_mode;        // 0 step, 1 linear
  u32 capture_index;
  u32 color_mode;          // 0 palette, 1 flow, 2 trap, 3 phase
  float flow_strength, flow_scale;
  u32 trap_kind, trap_mode;
  float trap_cx, trap_cy, trap_radius, trap_nx, trap_ny, trap_falloff, trap_freq, trap_strength;
  float phase_strength, phase_freq;
  float xform_blend;
  u64* counters;           // [0] accepted samples, [1] splats in bounds
  u64* sched;              // queue kernel: [0] walkers handed out, [1] fault flags
  u32* wrec;               // queue kernel: gridDim.x x QP walker records, 48 u32 each
  u32 cta_slots;           // queue kernel: slots filled per CTA at the start (<= QP)
};

// ---------------------------------------------------------------- seeding
// src/isaac.ts:194-229: PCG32 fills randrsl from (seed ^ hash(walker)),
// then irandinit(flag=1).  `w * 2654435761 + 1` is evaluated as a JS double
// before ToUint32, so it is computed in fp64 here for walkers >= 2^21.
VDEV void isaac_mix8(u32* v) {
  u32 a = v[0], b = v[1], c = v[2], d = v[3], e = v[4], f = v[5], g = v[6], h = v[7];
  a ^= b << 11; d += a; b += c;
  b ^= c >> 2;  e += b; c += d;
  c ^= d << 8;  f += c; d += e;
  d ^= e >> 16; g += d; e += f;
  e ^= f << 10; h += e; f += g;
  f ^= g >> 4;  a += f; g += h;
  g ^= h << 8;  b += g; h += a;
  h ^= a >> 9;  c += h; a += b;
  v[0] = a; v[1] = b; v[2] = c; v[3] = d; v[4] = e; v[5] = f; v[6] = g; v[7] = h;
}

VDEV u32 walker_hash(u64 w) {
  if (w < (1ull << 21)) return (u32)w * 2654435761u + 1u;
  // JS evaluates the product and the sum as two rounded doubles: no FMA.
  double d = __dadd_rn(__dmul_rn((double)w, 2654435761.0), 1.0);
  u64 q = (u64)d;
  return (u32)(q & 0xffffffffull);
}

// Out of line: once per walker, and large once unrolled.
OUTL void seed_walker_at(u32* s, u32 W, u32 seed, u64 w) {
  const Rng r{s, W};
  u32 pcg = seed ^ walker_hash(w);
#pragma unroll
  for (int k = 0; k < 4; ++k) pcg = pcg * 747796405u + 2891336453u;
  u32 v[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = 0x9e3779b9u;
#pragma unroll
  for (int i = 0; i < 4; ++i) isaac_mix8(v);
  u32 rsl[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    u32 s = pcg;
    pcg = pcg * 747796405u + 2891336453u;
    u32 word = ((s >> ((s >> 28) + 4u)) ^ s) * 277803737u;
    rsl[k] = (word >> 22) ^ word;
  }
  u32 mem[16];
#pragma unroll
  for (int i = 0; i < 16; i += 8) {
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] += rsl[i + j];
    isaac_mix8(v);
#pragma unroll
    for (int j = 0; j < 8; ++j) mem[i + j] = v[j];
  }
#pragma unroll
  for (int i = 0; i < 16; i += 8) {
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] += mem[i + j];
    isaac_mix8(v);
#pragma unroll
    for (int j = 0; j < 8; ++j) mem[i + j] = v[j];
  }
  r.f(1) = 0u; r.f(2) = 0u; r.f(3) = 0u;
#pragma unroll
  for (int k = 0; k < 16; ++k) { r.f(4 + k) = mem[k]; r.f(20 + k) = rsl[k]; }
  isaac_round(r);
  r.f(0) = 16u;
}
VDEV void seed_walker(const Rng& r, u32 seed, u64 w) { seed_walker_at(r.s, r.W, seed, w); }

// -------------------------------------------------------------- xform pick
// Row r of the reference's table (src/genome.ts:482-534) is nondecreasing
// in the grain index g, so table[r][g] = #{ j >= 1 : g >= start[r][j] }
// with start[r][j] = first g whose entry is >= j (16384 if none).  This
// reproduces the table bit for bit from NXF u16 per row.
VDEV u32 pick_xform(const unsigned short* st, u32 row, u32 g) {
  const unsigned short* s = st + row * NXF;
#if PICK_LINEAR
  u32 n = 0;
#pragma unroll
  for (int j = 1; j < NXF; ++j) n += (g >= (u32)s[j]) ? 1u : 0u;
  return n;
#else
  u32 lo = 0, hi = NXF - 1;  // answer in [lo, hi]; s[j] nondecreasing in j
  while (lo < hi) {
    u32 mid = (lo + hi + 1) >> 1;
    if (g >= (u32)s[mid]) lo = mid; else hi = mid - 1;
  }
  return lo;
#endif
}

// ------------------------------------------------------------------ splat
VDEV void add_sat(u32* cell, u32 delta) {
  if (delta == 0u) return;
  u32 old = atomicAdd(cell, delta);
  // Wrapped past 2^32 - 1: pin at the maximum.  Once any add overflows the
  // cell, every later add overflows again and re-pins, so the final value
  // is min(sum, 2^32 - 1) -- the saturating CAS result (chaos.wgsl:8120).
  if (old > 0xffffffffu - delta) atomicOr(cell, 0xffffffffu);
}

// Palette mix a*(1-t) + b*t with separately rounded products (no FMA), so
// the fixed-point deposit is bit-identical to the reference arithmetic.
VDEV float mix_rn(float a, float b, float t) {
  return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}

VDEV float3 mix3(float3 a, float3 b, float t) {
  return make_float3(mix_rn(a.x, b.x, t), mix_rn(a.y, b.y, t), mix_rn(a.z, b.z, t));
}

// The reference's affine row a*x + b*y + c, evaluated left to right with
// every product and sum rounded on its own.
VDEV float aff_rn(float a, float x, float b, float y, float c) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a, x), __fmul_rn(b, y)), c);
}

// (sin a, cos a) as the f32 roundings of the double-precision values: the
// correctly rounded f32 results except where a double result lies within
// one double ulp of an f32 rounding boundary.  Used by pre_blur, whose
// offsets then equal the reference's arithmetic bit for bit.
OUTL float2 sincos_rn(float a) {
  double s, c;
  sincos((double)a, &s, &c);
  return make_float2((float)s, (float)c);
}

// Scale-relative walker jitter (chaos.wgsl:8561-8565): v + (r - 0.5) * amp,
// each operation rounded on its own.
VDEV float jitter_rn(float v, float r, float amp) {
  return __fadd_rn(v, __fmul_rn(__fsub_rn(r, 0.5f), amp));
}

VDEV void splat(const ChaosArgs& A, const float4* pal, float3 sp, float2 p_start, float opacity,
                int dc_hit, float3 dc, u64* n_in) {
  // Bucket coordinates (chaos.wgsl:8575-8585), every product and sum rounded
  // on its own so the floor() boundaries match the reference exactly.
  float dx = __fsub_rn(sp.x, A.cx), dy = __fsub_rn(sp.y, A.cy);
  float rx = __fsub_rn(__fmul_rn(dx, A.cos_r), __fmul_rn(dy, A.sin_r));
  float ry = __fadd_rn(__fmul_rn(dx, A.sin_r), __fmul_rn(dy, A.cos_r));
  float px = __fadd_rn(__fmul_rn(rx, A.scale), __fmul_rn((float)A.width, 0.5f));
  float py = __fadd_rn(__fmul_rn(ry, A.scale), __fmul_rn((float)A.height, 0.5f));
  i32 xi = f2i(floorf(px)), yi = f2i(floorf(py));
  if (!(xi >= 0 && xi < (i32)A.width && yi >= 0 && yi < (i32)A.height)) return;
  *n_in += 1;
  float cxf = __fmul_rn(wclamp(sp.z, 0.0f, 1.0f), 255.0f);
  float4 pc;
  if (A.palette_mode == 1u) {
    u32 i0 = f2u(cxf);
    float fr = __fsub_rn(cxf, (float)i0);
    if (i0 >= 255u) { i0 = 254u; fr = 1.0f; }
    float4 a = pal[i0], b = pal[i0 + 1];
    pc = make_float4(mix_rn(a.x, b.x, fr), mix_rn(a.y, b.y, fr), mix_rn(a.z, b.z, fr), mix_rn(a.w, b.w, fr));
  } else {
    pc = pal[min(f2u(cxf), 255u)];
  }
  float3 rgb = make_float3(pc.x, pc.y, pc.z);
  if (dc_hit) rgb = dc;
  if (A.color_mode == 1u) {  // flow map, chaos.wgsl:8630-8650
    float2 d = f2(sp.x - p_start.x, sp.y - p_start.y);
    float mag = len2(d);
    if (mag > 1e-20f) {
      float hue = (atan2f(d.y, d.x) + P_PI) / (2.0f * P_PI);
      float val = wclamp(1.0f - expf(-fmaxf(A.flow_scale, 0.0f) * mag), 0.0f, 1.0f);
      rgb = mix3(rgb, hsv_rgb(hue, 1.0f, val), wclamp(A.flow_strength, 0.0f, 1.0f));
    }
  } else if (A.color_mode == 2u) {  // trap distance, chaos.wgsl:8656-8681
    float2 q = f2(sp.x - A.trap_cx, sp.y - A.trap_cy);
    float td = A.trap_kind == 0u ? len2(q)
             : (A.trap_kind == 1u ? fabsf(len2(q) - A.trap_radius) : fabsf(q.x * A.trap_nx + q.y * A.trap_ny));
    float tt = A.trap_mode == 0u ? wclamp(expf(-fmaxf(A.trap_falloff, 0.0f) * td), 0.0f, 1.0f)
                                 : wfract(td * fmaxf(A.trap_freq, 0.0f));
    float4 tp = pal[min(f2u(tt * 255.0f), 255u)];
    rgb = mix3(rgb, make_float3(tp.x, tp.y, tp.z), wclamp(A.trap_strength, 0.0f, 1.0f));
  } else if (A.color_mode == 3u) {  // phase / polar, chaos.wgsl:8689-8697
    float mag = len2(f2(sp.x, sp.y));
    if (mag > 1e-20f) {
      float hue = (atan2f(sp.y, sp.x) + P_PI) / (2.0f * P_PI);
      float ring = wfract(logf(mag) * fmaxf(A.phase_freq, 0.0f));
      rgb = mix3(rgb, hsv_rgb(hue, 1.0f, wmix(1.0f, 0.5f, ring)), wclamp(A.phase_strength, 0.0f, 1.0f));
    }
  }
  float wgt = __fmul_rn(opacity, 255.0f);
  u32* cell = A.hist + ((u64)yi * A.width + (u32)xi) * 4u;
  u32 dr = f2u(__fmul_rn(rgb.x, wgt)), dg = f2u(__fmul_rn(rgb.y, wgt)), db = f2u(__fmul_rn(rgb.z, wgt));
  u32 dn = f2u(wgt);
  // Warp aggregation.  Lanes whose deltas are below 2^26 may pool them (a
  // sum over 32 lanes then stays below 2^31, so pooling never wraps and the
  // saturating result min(total, 2^32 - 1) is unchanged).
  const u32 lane = threadIdx.x & 31u;
  const u32 act = __activemask();
  const u32 key = (u32)yi * A.width + (u32)xi;
  const bool small = ((dr | dg | db | dn) >> 26) == 0u;
  bool deposit = true;
#if AGGREGATE
  // Every distinct bucket of the warp deposits once (__match_any_sync).
  const u32 peers = __match_any_sync(act, small ? key : (0x80000000u | lane));
  if (__popc(peers) > 1) {
    dr = __reduce_add_sync(peers, dr);
    dg = __reduce_add_sync(peers, dg);
    db = __reduce_add_sync(peers, db);
    dn = __reduce_add_sync(peers, dn);
    deposit = lane == (u32)(__ffs(peers) - 1);
  }
#else
  // The hot bucket: lanes that hit the first eligible lane's bucket pool
  // their deltas.  Costs a shuffle and two ballots; turns the same-cell
  // atomic storm of a collapsing attractor into one deposit per warp.
  const u32 ok = __ballot_sync(act, small);
  if (ok) {
    const int lead = __ffs(ok) - 1;
    const u32 k0 = __shfl_sync(act, key, lead);
    const bool mine = small && key == k0;
    const u32 grp = __ballot_sync(act, mine);
    if (mine && __popc(grp) > 1) {
      dr = __reduce_add_sync(grp, dr);
      dg = __reduce_add_sync(grp, dg);
      db = __reduce_add_sync(grp, db);
      dn = __reduce_add_sync(grp, dn);
      deposit = lane == (u32)lead;
    }
  }
#endif
  if (deposit) {
    add_sat(cell + 0, dr);
    add_sat(cell + 1, dg);
    add_sat(cell + 2, db);
    add_sat(cell + 3, dn);
  }
  if (A.capture_index && A.idx_sum) {
    add_sat(A.idx_sum + (u64)yi * A.width + (u32)xi, f2u(__fmul_rn(wclamp(sp.z, 0.0f, 1.0f), wgt)));
  }
}

// ==== PYR3 KERNEL SECTION ====
// (the generator inserts xform_chain / final_chain above this line)

#ifndef QUEUE
#define QUEUE 0
#endif

// One xform chain of walker state p0/pz for xform k, with the optional
// xform blend (chaos.wgsl:8372-8381): with probability xform_blend a
// second xform's chain is mixed in.
VDEV void run_chain(const ChaosArgs& A, const unsigned short* pst, int k, float2 p0, float pz,
                    const Rng& rng, ChainOut& o) {
  Ctx cx;
  cx.rng = rng;
  const float* X = c_xf + k * 116;
  cx.a0 = make_float4(X[0], X[1], X[2], X[3]);
  cx.a1 = make_float4(X[4], X[5], X[6], X[7]);
  o.dc_hit = 0;
  o.dc = make_float3(0.0f, 0.0f, 0.0f);
  xform_chain(k, p0, pz, cx, o);
  if (A.xform_blend > 0.0f) {
    if (rand01(rng) < A.xform_blend) {
      u32 bi = pick_xform(pst, NXF, irand(rng) & 16383u);
      Ctx cb = cx;
      const float* XB = c_xf + bi * 116;
      cb.a0 = make_float4(XB[0], XB[1], XB[2], XB[3]);
      cb.a1 = make_float4(XB[4], XB[5], XB[6], XB[7]);
      ChainOut ob;
      ob.dc_hit = 0;
      ob.dc = make_float3(0.0f, 0.0f, 0.0f);
      xform_chain((int)bi, p0, pz, cb, ob);
      float tb = rand01(rng);
      o.pv = f2(mix_rn(o.pv.x, ob.pv.x, tb), mix_rn(o.pv.y, ob.pv.y, tb));
      o.nz = mix_rn(o.nz, ob.nz, tb);
    }
  }
}

VDEV bool bad_point(float2 v) {  // chaos.wgsl:8391: NaN or |v| > 1e10
  return (v.x != v.x) || (v.y != v.y) || fabsf(v.x) > 1e10f || fabsf(v.y) > 1e10f;
}

// Accepted iteration (chaos.wgsl:8455-8730) after the chain of xform fn
// produced pv / nz: final xform behind its opacity gate, scale-relative
// jitter of the walker position, and the splat once past the fuse.
// Returns the walker's next position.
VDEV float3 accept_step(const ChaosArgs& A, const float4* pal, const Rng& rng, int fn, float2 pv,
                        float nz, int dc_hit, float3 dc, float2 p_start, bool past_fuse,
                        u64* acc_samples, u64* acc_in) {
  float3 sp = make_float3(pv.x, pv.y, nz);
#if HAS_FINAL
  {
    const float* F = c_xf + FINAL_SLOT * 116;
    bool apply = true;
    if (F[10] != 1.0f) apply = rand01(rng) < F[10];
    // During the burn-in the final xform's output is not splatted; one that
    // draws nothing (and has no gate, which draws) need not run at all.
    else if (FINAL_RNG_FREE && !past_fuse) apply = false;
    if (apply) {
      Ctx cf;
      cf.rng = rng;
      cf.a0 = make_float4(F[0], F[1], F[2], F[3]);
      cf.a1 = make_float4(F[4], F[5], F[6], F[7]);
      ChainOut of;
      of.dc_hit = dc_hit;
      of.dc = dc;
      final_chain(pv, nz, cf, of);
      dc_hit = of.dc_hit;
      dc = of.dc;
      if (!bad_point(of.pv)) sp = make_float3(of.pv.x, of.pv.y, of.nz);
    }
  }
#endif
  const float mag = fmaxf(fmaxf(fabsf(pv.x), fabsf(pv.y)), 1e-30f);
  const float amp = mag * A.jitter;
  const float nx = jitter_rn(pv.x, rand01(rng), amp);
  const float ny = jitter_rn(pv.y, rand01(rng), amp);
  if (past_fuse) {
    *acc_samples += 1;
    splat(A, pal, sp, p_start, c_xf[fn * 116 + 10], dc_hit, dc, acc_in);
  }
  return make_float3(nx, ny, nz);
}

// One pass of the reference's iteration loop (chaos.wgsl:8330-8731) for a
// walker whose picked xform is k: the chain, the bad-value reseed with its
// retry count, and on acceptance the final xform, jitter and splat.  The
// walker state (position p, colour z, iteration index i, last accepted
// xform prev (-1: none), consecutive bad values) is updated in place.
VDEV void walker_iter(const ChaosArgs& A, const unsigned short* pst, const float4* pal,
                      const Rng& rng, int k, float2& p, float& z, u32& i, int& prev, u32& consec,
                      u64* acc_samples, u64* acc_in) {
  const float2 p_start = p;
  ChainOut o;
  run_chain(A, pst, k, p_start, z, rng, o);
  float2 pv = o.pv;
  const float nz = o.nz;
  if (bad_point(pv)) {
    const float bx = rand_11(rng);
    const float by = rand_11(rng);
    pv = f2(bx, by);
    consec += 1u;
  } else {
    consec = 0u;
  }
  float3 np = make_float3(pv.x, pv.y, nz);
  if (consec > 0u && consec < 5u) {
    if (i == 0u) i = 1u;  // the reference's rollback stops at 0
  } else {
    if (consec >= 5u) consec = 0u;
    prev = k;
    np = accept_step(A, pal, rng, k, pv, nz, o.dc_hit, o.dc, p_start, i >= A.fuse, acc_samples,
                     acc_in);
    i += 1u;
  }
  p = f2(np.x, np.y);
  z = np.z;
}

// --------------------------------------------------------------- kernel
extern "C" __global__ void __launch_bounds__(WPB)
chaos_kernel(const __grid_constant__ ChaosArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  u32* st = (u32*)smem;                                   // [36][WPB] ISAAC
  float4* pal = (float4*)(st + 36 * WPB);                 // [256]
  float* wx = (float*)(pal + 256);                        // walker point
  float* wy = wx + WPB;
  float* wz = wy + WPB;
  float* rx = wz + WPB;                                   // chain results
  float* ry = rx + WPB;
  float* rz = ry + WPB;
  float* dcr = rz + WPB;
  float* dcg = dcr + WPB;
  float* dcb = dcg + WPB;
  int* wfn = (int*)(dcb + WPB);                           // picked xform
  int* dch = wfn + WPB;                                   // dc hit flag
  unsigned short* order = (unsigned short*)(dch + WPB);   // slot -> walker
  unsigned short* pst = order + WPB;                      // pick boundaries
  int* bucket = (int*)(pst + ((MAXRANK * NXF + 1) & ~1)); // NXF + 2 counters

  const u32 t = threadIdx.x;
  for (u32 i = t; i < 256u; i += WPB) pal[i] = ((const float4*)A.palette)[i];
  for (u32 k = t; k < (u32)(NXF + 2); k += WPB) bucket[k] = 0;
  for (u32 i = t; i < (u32)(MAXRANK * NXF); i += WPB) pst[i] = A.pick_start[i];

  const u64 sets = (A.n_walkers + WPB - 1) / WPB;
  u64 acc_samples = 0, acc_in = 0;
  for (u64 set = blockIdx.x; set < sets; set += gridDim.x) {
    const u64 lw = set * WPB + t;             // walker index within the launch
    const bool real = lw < A.n_walkers;
    const u64 gw = A.walker_base + lw;
    Rng rng{st + t, WPB};
    u64 total = 0;
    if (real) {
      total = A.iters_base + (lw < A.iters_extra ? 1ull : 0ull) + A.fuse;
      seed_walker(rng, A.seed, gw);
      float x0 = rand_11(rng);
      float y0 = rand_11(rng);
      float z0 = rand01(rng);
      wx[t] = x0; wy[t] = y0; wz[t] = z0;
    }
    int prev = -1;
    u32 consec_bad = 0;
    u64 i = 0;
    __syncthreads();
    while (__syncthreads_or(i < total)) {
      // ---- phase A: pick + bucket
      for (u32 k = t; k < (u32)(NXF + 2); k += WPB) bucket[k] = 0;
      __syncthreads();
      const bool active = i < total;
      int fn = NXF;  // inactive walkers go to the sentinel bucket
      if (active) {
        u32 row = prev >= 0 ? (u32)prev : (u32)NXF;
        fn = (int)pick_xform(pst, row, irand(rng) & 16383u);
      }
      wfn[t] = fn;
      const int rank = atomicAdd(&bucket[fn], 1);
      __syncthreads();
      if (t < 32) {  // exclusive scan of the NXF+1 bucket counts
        int carry = 0;
        for (int base = 0; base < NXF + 1; base += 32) {
          int k = base + (int)t;
          int v = k < NXF + 1 ? bucket[k] : 0;
          int incl = v;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            int n = __shfl_up_sync(0xffffffffu, incl, o);
            if ((int)t >= o) incl += n;
          }
          if (k < NXF + 1) bucket[k] = carry + incl - v;
          carry += __shfl_sync(0xffffffffu, incl, 31);
        }
      }
      __syncthreads();
      order[bucket[fn] + rank] = (unsigned short)t;
      const int n_act = bucket[NXF];
      __syncthreads();
      // ---- phase B: xform chains in xform order
      if ((int)t < n_act) {
        const u32 w = order[t];
        const int k = wfn[w];
        Ctx cx;
        cx.rng = Rng{st + w, WPB};
        const float* X = c_xf + k * 116;
        cx.a0 = make_float4(X[0], X[1], X[2], X[3]);
        cx.a1 = make_float4(X[4], X[5], X[6], X[7]);
        ChainOut o;
        o.dc_hit = 0;
        o.dc = make_float3(0.0f, 0.0f, 0.0f);
        const float2 p0 = f2(wx[w], wy[w]);
        const float pz = wz[w];
        xform_chain(k, p0, pz, cx, o);
        if (A.xform_blend > 0.0f) {  // chaos.wgsl:8372-8381
          if (rand01(cx.rng) < A.xform_blend) {
            u32 bi = pick_xform(pst, NXF, irand(cx.rng) & 16383u);
            Ctx cb = cx;
            const float* XB = c_xf + bi * 116;
            cb.a0 = make_float4(XB[0], XB[1], XB[2], XB[3]);
            cb.a1 = make_float4(XB[4], XB[5], XB[6], XB[7]);
            ChainOut ob;
            ob.dc_hit = 0;
            ob.dc = make_float3(0.0f, 0.0f, 0.0f);
            xform_chain((int)bi, p0, pz, cb, ob);
            float tb = rand01(cx.rng);
            o.pv = f2(mix_rn(o.pv.x, ob.pv.x, tb), mix_rn(o.pv.y, ob.pv.y, tb));
            o.nz = mix_rn(o.nz, ob.nz, tb);
          }
        }
        rx[w] = o.pv.x; ry[w] = o.pv.y; rz[w] = o.nz;
        dcr[w] = o.dc.x; dcg[w] = o.dc.y; dcb[w] = o.dc.z; dch[w] = o.dc_hit;
      }
      __syncthreads();
      // ---- phase C: retry logic, final xform, jitter, splat
      if (active) {
        float2 pv = f2(rx[t], ry[t]);
        float nz = rz[t];
        const float2 p_start = f2(wx[t], wy[t]);
        const bool bad = (pv.x != pv.x) || (pv.y != pv.y) || fabsf(pv.x) > 1e10f || fabsf(pv.y) > 1e10f;
        if (bad) {
          float sx = rand_11(rng);
          float sy = rand_11(rng);
          pv = f2(sx, sy);
          consec_bad += 1u;
        } else {
          consec_bad = 0u;
        }
        if (consec_bad > 0u && consec_bad < 5u) {
          wx[t] = pv.x; wy[t] = pv.y; wz[t] = nz;
          if (i == 0) i = 1;  // the reference's rollback stops at 0
        } else {
          if (consec_bad >= 5u) consec_bad = 0u;
          prev = fn;
          float3 sp = make_float3(pv.x, pv.y, nz);
          int dc_hit = dch[t];
          float3 dc = make_float3(dcr[t], dcg[t], dcb[t]);
#if HAS_FINAL
          {
            const float* F = c_xf + FINAL_SLOT * 116;
            bool apply = true;
            if (F[10] != 1.0f) apply = rand01(rng) < F[10];
            else if (FINAL_RNG_FREE && i < A.fuse) apply = false;  // not splatted, draws nothing
            if (apply) {
              Ctx cf;
              cf.rng = rng;
              cf.a0 = make_float4(F[0], F[1], F[2], F[3]);
              cf.a1 = make_float4(F[4], F[5], F[6], F[7]);
              ChainOut of;
              of.dc_hit = dc_hit;
              of.dc = dc;
              final_chain(pv, nz, cf, of);
              dc_hit = of.dc_hit;
              dc = of.dc;
              const bool fbad = (of.pv.x != of.pv.x) || (of.pv.y != of.pv.y) ||
                                fabsf(of.pv.x) > 1e10f || fabsf(of.pv.y) > 1e10f;
              if (!fbad) sp = make_float3(of.pv.x, of.pv.y, of.nz);
            }
          }
#endif
          const float mag = fmaxf(fmaxf(fabsf(pv.x), fabsf(pv.y)), 1e-30f);
          const float amp = mag * A.jitter;
          const float jx = jitter_rn(pv.x, rand01(rng), amp);
          const float jy = jitter_rn(pv.y, rand01(rng), amp);
          wx[t] = jx; wy[t] = jy; wz[t] = nz;
          if (i >= A.fuse) {
            acc_samples += 1;
            splat(A, pal, sp, p_start, c_xf[fn * 116 + 10], dc_hit, dc, &acc_in);
          }
          i += 1;
        }
      }
    }
  }
  if (A.counters) {
    atomicAdd(&A.counters[0], acc_samples);
    atomicAdd(&A.counters[1], acc_in);
  }
}

#if QUEUE
// ------------------------------------------------------------ queue kernel
// Compiled beside chaos_kernel for genomes of up to 32 xforms; the host
// picks one of the two per launch.  One CTA per SM owns QP walker slots.
// Their records (ISAAC state, point, counters) live in global memory,
// private to the CTA and small enough to stay in L2; the slot ids wait in
// one shared-memory ring per xform.  A warp takes up to 32 slots from one
// ring, stages their records in shared memory, runs one iteration of each
// -- its lanes execute that xform's chain together -- writes the records
// back and pushes every slot onto the ring of the xform its walker picked
// next.  Warps never wait for one another at a barrier.  The warps of a
// CTA keep to the CTA's current ring while it holds a full batch, so an SM
// runs one xform's code at a time and the instruction working set stays
// small however many xforms the genome has; keeping only the ring entries
// on chip is what lets a CTA hold enough walkers for that.
//
// The next pick is drawn at the end of an iteration from the walker's own
// stream -- the first draw of its next iteration, where the reference
// draws it.  A finished walker's slot is reseeded with the next walker of
// the launch (sched[0] counts walkers handed out) or retired.
//
// Rings: QP cells of u16 each; a ring never holds more than QP entries
// because each slot is in at most one ring; head and tail only grow.  A
// cell is FREE(lap) = lap << 11 or FULL(lap, slot) = 0x8000 | lap << 11 |
// slot, lap = (position / QP) mod 16.  A producer reserves a position with
// atomicAdd on tail, waits for FREE(lap) there and writes FULL(lap, slot);
// a consumer reserves positions with atomicCAS on head, waits for
// FULL(lap), takes the slot and writes FREE(lap + 1).  The cell a producer
// waits for was reserved by a consumer one lap earlier (a ring would
// otherwise hold more than QP slots), so every wait ends; each is bounded
// all the same, and past the limit the kernel sets sched[1] and returns,
// which the host reports.
//
// Records are only ever touched by their own CTA, so CTA-scope fences order
// a record's write-back before its slot is pushed, and a slot's take before
// its record is read; the record traffic bypasses L1 (ld/st .cg).
#define QP 2048                // walker slots per CTA (slot ids fit 11 bits)
#define QP_LOG2 11
#define QFULL 0x8000u
#define WR_WORDS 48            // record stride in u32 (192 B)
#define WR_PARTS 11            // uint4 parts that carry data (words 0..43)
#define QSTAGE (44 * SST + 32)  // staging words per warp: 44 rows of SST, then the lanes' slots
#define SST 33                 // staging stride between ISAAC fields: conflict-free
#define QSPIN_LIMIT (1u << 22)
#define QIDLE_CYCLES 4000000000ll  // ~2 s at 1.97 GHz without work while walkers are live

// Bounded wait for cell c to satisfy (v & mask) == want; returns the value
// seen, or 0xffffffff after QSPIN_LIMIT polls.
VDEV u32 q_wait(volatile unsigned short* c, u32 mask, u32 want) {
  for (u32 spins = 0; spins < QSPIN_LIMIT; ++spins) {
    const u32 v = *c;
    if ((v & mask) == want) return v;
  }
  return 0xffffffffu;
}
// Append slot s at ring position pos; false on a timed-out wait.
VDEV bool q_put(unsigned short* ring_k, u32 pos, u32 s) {
  volatile unsigned short* c = ring_k + (pos & (QP - 1));
  const u32 lap = (pos >> QP_LOG2) & 15u;
  if (q_wait(c, 0xffffu, lap << 11) == 0xffffffffu) return false;
  *c = (unsigned short)(QFULL | (lap << 11) | s);
  return true;
}
// Take the slot at ring position pos; false on a timed-out wait.
VDEV bool q_take(unsigned short* ring_k, u32 pos, u32* s) {
  volatile unsigned short* c = ring_k + (pos & (QP - 1));
  const u32 lap = (pos >> QP_LOG2) & 15u;
  const u32 v = q_wait(c, 0xf800u, QFULL | (lap << 11));
  if (v == 0xffffffffu) return false;
  *s = v & (QP - 1);
  *c = (unsigned short)(((lap + 1u) & 15u) << 11);
  return true;
}
VDEV u32 vld(const u32* p) { return *(const volatile u32*)p; }

// Staged walker of lane `lane`: ISAAC fields at sst[k * SST + lane]; record
// words 36..41 at sf[(w - 36) * SST + lane]: x, y, z bits, iteration index,
// fuse + iterations, prev xform (low byte, 0xff = none) | bad count << 8.
// Seed walker lw of the launch into it (src/isaac.ts:194-229) and draw its
// start point (chaos.wgsl:8302-8305).
VDEV void q_seed(const ChaosArgs& A, u32* sst, u32* sf, u32 lane, u64 lw) {
  const Rng r{sst + lane, SST};
  seed_walker(r, A.seed, A.walker_base + lw);
  const float x0 = rand_11(r);
  const float y0 = rand_11(r);
  const float z0 = rand01(r);
  sf[lane] = __float_as_uint(x0);
  sf[SST + lane] = __float_as_uint(y0);
  sf[2 * SST + lane] = __float_as_uint(z0);
  sf[3 * SST + lane] = 0u;
  sf[4 * SST + lane] = (u32)(A.iters_base + (lw < A.iters_extra ? 1ull : 0ull) + A.fuse);
  sf[5 * SST + lane] = 0xffu;
}
// Record <-> staging for the first n lanes' slots in ssl (coalesced): lane
// q moves 16-byte part j = q % WR_PARTS of record r = q / WR_PARTS, whose
// four words sit in staging rows 4j..4j+3 (rows 42 and 43 are padding).
VDEV void q_load(const ChaosArgs& A, const u32* ssl, u32 n, u32 lane, u32* sst) {
  const u32* base = A.wrec + (u64)blockIdx.x * QP * WR_WORDS;
  for (u32 q = lane; q < n * WR_PARTS; q += 32u) {
    const u32 r = q / WR_PARTS, j = q - r * WR_PARTS;
    const uint4 v = __ldcg((const uint4*)(base + (u64)ssl[r] * WR_WORDS) + j);
    u32* d = sst + j * (4u * SST) + r;
    d[0] = v.x;
    d[SST] = v.y;
    d[2 * SST] = v.z;
    d[3 * SST] = v.w;
  }
}
VDEV void q_store(const ChaosArgs& A, const u32* ssl, u32 n, u32 lane, const u32* sst) {
  u32* base = A.wrec + (u64)blockIdx.x * QP * WR_WORDS;
  for (u32 q = lane; q < n * WR_PARTS; q += 32u) {
    const u32 r = q / WR_PARTS, j = q - r * WR_PARTS;
    const u32* d = sst + j * (4u * SST) + r;
    __stcg((uint4*)(base + (u64)ssl[r] * WR_WORDS) + j, make_uint4(d[0], d[SST], d[2 * SST], d[3 * SST]));
  }
}

extern "C" __global__ void __launch_bounds__(QWARPS * 32, 1)
chaos_queue_kernel(const __grid_constant__ ChaosArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  float4* pal = (float4*)smem;                                  // [256]
  u32* stage = (u32*)(pal + 256);                               // [QWARPS][QSTAGE]
  unsigned short* ring = (unsigned short*)(stage + QWARPS * QSTAGE);  // [NXF][QP]
  unsigned short* pst = ring + NXF * QP;                        // pick boundaries
  u32* qhead = (u32*)(pst + ((MAXRANK * NXF + 1) & ~1));
  u32* qtail = qhead + NXF;
  int* live = (int*)(qtail + NXF);
  u32* aff = (u32*)(live + 1);                                  // the CTA's current ring

  const u32 t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  for (u32 i = t; i < 256u; i += blockDim.x) pal[i] = ((const float4*)A.palette)[i];
  for (u32 i = t; i < (u32)(MAXRANK * NXF); i += blockDim.x) pst[i] = A.pick_start[i];
  for (u32 i = t; i < (u32)(NXF * QP); i += blockDim.x) ring[i] = 0;  // FREE(lap 0)
  if (t < (u32)NXF) { qhead[t] = 0u; qtail[t] = 0u; }
  if (t == 0) { *live = 0; *aff = 0u; }
  __syncthreads();
  u32* sst = stage + warp * QSTAGE;
  u32* sf = sst + 36 * SST;                                     // record words 36.. (stride SST)
  u32* ssl = sst + 44 * SST;                                    // slot of each lane

  // ---- fill the slots, 32 at a time per warp
  for (u32 b = warp * 32u; b < A.cta_slots; b += QWARPS * 32u) {
    const u32 s = b + lane;
    bool have = false;
    u32 fn = 0u;
    if (s < A.cta_slots) {
      const u64 lw = atomicAdd((unsigned long long*)&A.sched[0], 1ull);
      if (lw < A.n_walkers) {
        q_seed(A, sst, sf, lane, lw);
        fn = pick_xform(pst, NXF, irand(Rng{sst + lane, SST}) & 16383u);
        have = true;
      }
    }
    ssl[lane] = s;
    __syncwarp();
    // Store every lane whose slot exists (a prefix of the warp); slots that
    // got no walker are never queued, so their records are never read.
    const u32 nb = A.cta_slots - b < 32u ? A.cta_slots - b : 32u;
    q_store(A, ssl, nb, lane, sst);
    __threadfence_block();
    __syncwarp();
    if (have) {
      const u32 pos = atomicAdd(&qtail[fn], 1u);  // fewer than QP so far: lap 0, cell FREE(0)
      ring[fn * QP + (pos & (QP - 1))] = (unsigned short)(QFULL | s);
      atomicAdd(live, 1);
    }
    __syncwarp();
  }
  __syncthreads();

  u64 acc_samples = 0, acc_in = 0;
  long long idle_since = -1;
  bool fault = false;
  while (!fault) {
    // ---- choose a ring: the CTA's current one while it holds a full batch
    u32 k = *(volatile u32*)aff;
    const u32 hk = vld(&qhead[k]);
    const u32 len = vld(&qtail[k]) - hk;
    if (len < 32u) {  // else the longest ring (ties: lowest xform)
      u32 l2 = 0u;
      if (lane < (u32)NXF) {
        const u32 hh = vld(&qhead[lane]);  // head first: tail >= head at any later time
        l2 = vld(&qtail[lane]) - hh;
      }
      u32 best = l2, bk = lane;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const u32 ol = __shfl_xor_sync(0xffffffffu, best, o);
        const u32 ok = __shfl_xor_sync(0xffffffffu, bk, o);
        if (ol > best || (ol == best && ok < bk)) { best = ol; bk = ok; }
      }
      if (best == 0u) {
        if (*(volatile int*)live == 0) break;
        const long long now = clock64();
        if (idle_since < 0) idle_since = now;
        else if (now - idle_since > QIDLE_CYCLES) { fault = true; break; }
        __nanosleep(64);
        continue;
      }
      k = bk;
      if (lane == 0) *(volatile u32*)aff = k;
    }
    idle_since = -1;
    // ---- reserve up to 32 positions of ring k
    u32 h = 0u, n = 0u;
    if (lane == 0) {
      h = vld(&qhead[k]);
      const u32 avail = vld(&qtail[k]) - h;
      n = avail < 32u ? avail : 32u;
      if (n > 0u && atomicCAS(&qhead[k], h, h + n) != h) n = 0u;
    }
    n = __shfl_sync(0xffffffffu, n, 0);
    if (n == 0u) continue;
    h = __shfl_sync(0xffffffffu, h, 0);
    // ---- take the slots and stage their records
    if (lane < n) {
      u32 s = 0u;
      if (q_take(ring + k * QP, h + lane, &s)) ssl[lane] = s;
      else fault = true;
    }
    if (__any_sync(0xffffffffu, fault)) { fault = true; break; }
    __syncwarp();
    __threadfence_block();
    q_load(A, ssl, n, lane, sst);
    __syncwarp();

    // ---- one iteration of each staged walker (the warp runs xform k)
    bool push = false;
    u32 nfn = 0u;
    if (lane < n) {
      const Rng rng{sst + lane, SST};
      float2 p = f2(__uint_as_float(sf[lane]), __uint_as_float(sf[SST + lane]));
      float z = __uint_as_float(sf[2 * SST + lane]);
      u32 i = sf[3 * SST + lane];
      const u32 pb = sf[5 * SST + lane];
      u32 consec = pb >> 8;
      int prev = (int)(pb & 0xffu);
      if (prev == 0xff) prev = -1;
      walker_iter(A, pst, pal, rng, (int)k, p, z, i, prev, consec, &acc_samples, &acc_in);
      sf[lane] = __float_as_uint(p.x);
      sf[SST + lane] = __float_as_uint(p.y);
      sf[2 * SST + lane] = __float_as_uint(z);
      sf[3 * SST + lane] = i;
      sf[5 * SST + lane] = ((u32)prev & 0xffu) | (consec << 8);
      push = true;
      if (i >= sf[4 * SST + lane]) {  // finished: the next walker of the launch, or retire the slot
        const u64 lw = atomicAdd((unsigned long long*)&A.sched[0], 1ull);
        if (lw < A.n_walkers) {
          q_seed(A, sst, sf, lane, lw);
          prev = -1;
        } else {
          atomicSub(live, 1);
          push = false;
        }
      }
      if (push) nfn = pick_xform(pst, prev >= 0 ? (u32)prev : (u32)NXF, irand(rng) & 16383u);
    }
    __syncwarp();
    // ---- write the records back, then push the slots
    q_store(A, ssl, n, lane, sst);
    __threadfence_block();
    __syncwarp();
    const u32 pm = __ballot_sync(0xffffffffu, push);
    if (push) {
      const u32 peers = __match_any_sync(pm, nfn);
      const u32 leader = (u32)(__ffs(peers) - 1);
      u32 base = 0u;
      if (lane == leader) base = atomicAdd(&qtail[nfn], (u32)__popc(peers));
      base = __shfl_sync(peers, base, leader);
      const u32 rank = (u32)__popc(peers & ((1u << lane) - 1u));
      if (!q_put(ring + nfn * QP, base + rank, ssl[lane])) fault = true;
    }
    fault = __any_sync(0xffffffffu, fault);
    __syncwarp();
  }
  if (fault && lane == 0) atomicOr((unsigned long long*)&A.sched[1], 1ull);
  if (A.counters) {
    atomicAdd(&A.counters[0], acc_samples);
    atomicAdd(&A.counters[1], acc_in);
  }
}
#endif  // QUEUE

#ifndef WAVE
#define WAVE 0
#endif
#if WAVE
// --------------------------------------------------------- wave kernel
// Bulk-synchronous alternative for large launches: every walker of the
// launch is resident in global memory, grouped by the xform it runs next,
// and each launch of chaos_wave_kernel advances every walker by one
// iteration.  Block b takes the b-th chunk of WB walkers in region order
// (xform 0's chunks first), so all of a block's walkers run one xform --
// full warps on one xform's straight-line code -- and the blocks resident
// on the GPU at any moment run one or two xforms, which keeps the
// instruction working set small.  After the iteration each block counting-
// sorts its walkers by their next xform in shared memory, reserves room in
// the next buffer's regions with one atomicAdd per xform, and writes the
// walkers out in sorted order (coalesced).  No block ever waits on another.
// The host sizes the pool so both populations' records fit in half of L2;
// records are written with an evict-last policy and dropped from L2 once
// copied in, so between launches they need not touch HBM, which is left to
// the histogram's atomics.
//
// State: st[2][NXF][WF][cap] u32 (two buffers, field-major so a chunk's
// field is one contiguous 1 KB line) -- fields 0..42 the ISAAC state in the
// Rng layout with the early-refill stash, then x, y, z bits, iteration
// index, iterations to run (fuse included), last accepted xform (low byte,
// 0xff = none) | bad count << 8.
//
// ISAAC rounds: a walker needs one per 16 draws, and a draw site where any
// lane of a warp runs dry makes the whole warp wait for that lane's round.
// Each iteration therefore starts with isaac_early_refill: walkers with
// fewer than 8 unread results move them to the stash and run the round
// there, together, so a warp runs one round per iteration instead of one
// per draw site.  The stream of values is unchanged.
// Walker counts per region: cnt[3][NXF]; a launch reads cnt[rd_cnt], adds
// into cnt[wr_cnt] and zeroes cnt[zero_cnt] for the launch after next.
// Modes: 0 seeds walkers [b*WB, b*WB + WB) and sorts them by first pick;
// 1 runs one iteration; 2 (the last launch) runs each remaining walker to
// its end in place -- walkers still running after the planned launches are
// the ones whose bad-value retries did not count as iterations.
#define WB 256
#define WF 49                  // state words per walker
#define WRNG 43                // of which ISAAC state + stash (shared-memory rows)

struct WaveArgs {
  u32* st;
  u32* cnt;
  u64 cap;        // walkers per region (>= walkers in the launch)
  u32 mode;
  u32 rd_buf, wr_buf;
  u32 rd_cnt, wr_cnt, zero_cnt;
};

// Refill a walker's ISAAC block before it runs dry: with fewer than 8
// results unread (and no stash in use) stash them, run the round, and mark
// the new block full (cnt 16).
VDEV void isaac_early_refill(const Rng& r) {
  const u32 c = r.f(0);
  if (c < 8u) {
#pragma unroll
    for (u32 j = 0; j < 7u; ++j)
      if (j < c) r.f(36 + j) = r.f(20 + j);
    isaac_round(r);
    r.f(0) = (c << 8) | 16u;
  }
}

VDEV u32* wave_field(const WaveArgs& W, u32 buf, u32 k, u32 f) {
  return W.st + (((u64)buf * NXF + k) * WF + f) * W.cap;
}

// Bulk asynchronous copies (cp.async.bulk, no multicast) of a chunk's
// fields into shared memory, completing on one mbarrier.  Every source
// and destination is 1 KB aligned and every size a multiple of 16 bytes.
#define WAVE_WAIT_LIMIT (1u << 24)
VDEV u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }
VDEV void mbar_init(u64* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n"
               "fence.mbarrier_init.release.cluster;\n" ::"r"(smem_u32(bar)) : "memory");
}
VDEV void mbar_expect_tx(u64* bar, u32 bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n"
               ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
VDEV void bulk_g2s(void* dst, const void* src, u32 bytes, u64* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// 4-byte store cached in L2 only (st.global.cg) under L2 cache policy pol.
VDEV void st_keep(u32* dst, u32 v, u64 pol) {
  asm volatile("st.global.cg.L2::cache_hint.b32 [%0], %1, %2;" ::"l"(dst), "r"(v), "l"(pol) : "memory");
}
// Wait for phase 0 of the barrier; false if WAVE_WAIT_LIMIT polls pass.
VDEV bool mbar_wait0(u64* bar) {
  for (u32 it = 0; it < WAVE_WAIT_LIMIT; ++it) {
    u32 done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n" : "=r"(done) : "r"(smem_u32(bar)) : "memory");
    if (done) return true;
  }
  return false;
}

extern "C" __global__ void __launch_bounds__(WB, WAVE_MINB)
chaos_wave_kernel(const __grid_constant__ ChaosArgs A, const __grid_constant__ WaveArgs W) {
  extern __shared__ __align__(16) unsigned char smem[];
  float4* pal = (float4*)smem;                                  // [256]
  u32* srng = (u32*)(pal + 256);                                // [WRNG][WB]
  u32* sfs = srng + WRNG * WB;                                  // [6][WB] walker fields
  u32* sdst = sfs + 6 * WB;                                     // [WB] destination of sorted slot
  u32* scnt = sdst + WB;                                        // [NXF] walkers per next xform
  u32* soff = scnt + NXF;                                       // [NXF + 1] sorted offsets
  u32* sbase = soff + NXF + 1;                                  // [NXF] region positions
  u32* swork = sbase + NXF;                                     // [3] xform, chunk, region count
  unsigned short* sperm = (unsigned short*)(swork + 3);         // [WB] walker of sorted slot
  unsigned char* skey = (unsigned char*)(sperm + WB);           // [WB] its next xform
  unsigned short* pst = (unsigned short*)(skey + WB);           // pick boundaries

  __shared__ __align__(8) u64 wbar;

  const u32 t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  if (W.mode == 0u)
    for (u32 i = t; i < 256u; i += WB) pal[i] = ((const float4*)A.palette)[i];
  else if (t == 0)
    mbar_init(&wbar);
  for (u32 i = t; i < (u32)(MAXRANK * NXF); i += WB) pst[i] = A.pick_start[i];
  if (blockIdx.x == 0 && t < (u32)NXF && W.mode != 2u) W.cnt[W.zero_cnt * NXF + t] = 0u;
  if (t < (u32)NXF) scnt[t] = 0u;  // sort counts, first used after the iteration
  if (W.mode != 0u && warp == 0) {
    // This block's work item: chunk c of region k, regions in xform order.
    const u32 c = lane < (u32)NXF ? W.cnt[W.rd_cnt * NXF + lane] : 0u;
    const u32 nb = (c + WB - 1u) / WB;
    u32 incl = nb;
#pragma unroll
    for (u32 o = 1; o < 32u; o <<= 1) {
      const u32 v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const u32 m = __ballot_sync(0xffffffffu, incl > blockIdx.x);
    const u32 k = m ? (u32)(__ffs(m) - 1) : 0u;
    const u32 first = __shfl_sync(0xffffffffu, incl - nb, k);
    const u32 ck = __shfl_sync(0xffffffffu, c, k);
    if (lane == 0) {
      swork[0] = m ? k : 0xffffffffu;
      swork[1] = blockIdx.x - first;
      swork[2] = ck;
    }
  }
  __syncthreads();
  const Rng rng{srng + t, WB};
  u64 acc_samples = 0, acc_in = 0;
  bool alive = false;
  u32 nfn = 0u;
  float2 p = f2(0.0f, 0.0f);
  float z = 0.0f;
  u32 i = 0u, iters = 0u, consec = 0u;
  int prev = -1;
  if (W.mode == 0u) {
    const u64 lw = (u64)blockIdx.x * WB + t;
    if (lw < A.n_walkers) {
      seed_walker(rng, A.seed, A.walker_base + lw);
      const float x0 = rand_11(rng);
      const float y0 = rand_11(rng);
      z = rand01(rng);
      p = f2(x0, y0);
      iters = (u32)(A.iters_base + (lw < A.iters_extra ? 1ull : 0ull) + A.fuse);
      nfn = pick_xform(pst, (u32)NXF, irand(rng) & 16383u);
      alive = true;
    }
  } else {
    const u32 k = swork[0];
    if (k == 0xffffffffu) return;  // uniform: past the end of the work list
    const u32 pos0 = swork[1] * WB, pos = pos0 + t;
    // One thread moves the chunk (WF fields x 1 KB) and the palette into
    // shared memory; the chunk may extend past the region's walkers, never
    // past its capacity.  Bulk copies need 16-byte aligned sources: the host
    // lays the state out so they are, and a layout that is not is reported
    // (sched[1] bit 2), not copied.
    if (t == 0) {
      const bool aligned =
          ((reinterpret_cast<unsigned long long>(wave_field(W, W.rd_buf, k, 0) + pos0) |
            reinterpret_cast<unsigned long long>(A.palette) | (W.cap * 4ull)) & 15ull) == 0ull;
      sbase[0] = aligned ? 1u : 0u;  // flag (sbase is free until the sort)
      if (aligned) {
        mbar_expect_tx(&wbar, (u32)(WF * WB * 4 + 256 * 16));
        for (u32 f = 0; f < (u32)WRNG; ++f)
          bulk_g2s(srng + f * WB, wave_field(W, W.rd_buf, k, f) + pos0, WB * 4, &wbar);
        for (u32 f = 0; f < 6u; ++f)
          bulk_g2s(sfs + f * WB, wave_field(W, W.rd_buf, k, WRNG + f) + pos0, WB * 4, &wbar);
        bulk_g2s(pal, A.palette, 256 * 16, &wbar);
      } else {
        atomicOr((unsigned long long*)&A.sched[1], 4ull);
      }
    }
    __syncthreads();
    if (sbase[0] == 0u) return;  // uniform: misaligned layout, nothing copied
    if (!__syncthreads_and(mbar_wait0(&wbar))) {
      // The copy did not land in time (the whole block agrees): report it,
      // wait once more (bounded) so no copy is still writing this block's
      // shared memory, and drop the chunk.
      if (t == 0) atomicOr((unsigned long long*)&A.sched[1], 2ull);
      mbar_wait0(&wbar);
      return;
    }
    // The chunk's source lines are dead once copied: this launch reads each
    // chunk once, and the buffer is next read after the following launch has
    // rewritten it.  Dropping them from L2 (no write-back) keeps the records
    // of both populations L2-resident between launches.  Every field's chunk
    // is 1 KB aligned in the host layout; lines are dropped only where the
    // 128-byte alignment the instruction needs holds.
    if (((reinterpret_cast<unsigned long long>(wave_field(W, W.rd_buf, k, 0) + pos0) | (W.cap * 4ull)) &
         127ull) == 0ull) {
      for (u32 q = t; q < (u32)WF * 8u; q += WB) {
        const u32* src = wave_field(W, W.rd_buf, k, q >> 3) + pos0 + (q & 7u) * 32u;
        asm volatile("discard.global.L2 [%0], 128;" ::"l"(src) : "memory");
      }
    }
    if (pos < swork[2]) {
      p = f2(__uint_as_float(sfs[t]), __uint_as_float(sfs[WB + t]));
      z = __uint_as_float(sfs[2 * WB + t]);
      i = sfs[3 * WB + t];
      iters = sfs[4 * WB + t];
      const u32 pb = sfs[5 * WB + t];
      consec = pb >> 8;
      prev = (pb & 0xffu) == 0xffu ? -1 : (int)(pb & 0xffu);
      // Mode 1: one iteration and the next pick; mode 2: to the walker's end.
      u32 kk = k;
      for (;;) {
        isaac_early_refill(rng);
        walker_iter(A, pst, pal, rng, (int)kk, p, z, i, prev, consec, &acc_samples, &acc_in);
        if (i >= iters) break;
        kk = pick_xform(pst, prev >= 0 ? (u32)prev : (u32)NXF, irand(rng) & 16383u);
        if (W.mode == 1u) {
          nfn = kk;
          alive = true;
          break;
        }
      }
    }
  }
  if (A.counters) {
    const u32 ds = __reduce_add_sync(0xffffffffu, (u32)acc_samples);
    const u32 di = __reduce_add_sync(0xffffffffu, (u32)acc_in);
    if (lane == 0) {
      if (ds) atomicAdd(&A.counters[0], (u64)ds);
      if (di) atomicAdd(&A.counters[1], (u64)di);
    }
  }
  if (W.mode == 2u) return;

  // ---- sort by next xform, reserve region space, write out
  u32 rank = 0u;
  if (alive) {
    rank = atomicAdd(&scnt[nfn], 1u);
    sfs[t] = __float_as_uint(p.x);
    sfs[WB + t] = __float_as_uint(p.y);
    sfs[2 * WB + t] = __float_as_uint(z);
    sfs[3 * WB + t] = i;
    sfs[4 * WB + t] = iters;
    sfs[5 * WB + t] = ((u32)prev & 0xffu) | (consec << 8);
  }
  __syncthreads();
  if (warp == 0) {
    const u32 c = lane < (u32)NXF ? scnt[lane] : 0u;
    u32 incl = c;
#pragma unroll
    for (u32 o = 1; o < 32u; o <<= 1) {
      const u32 v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane < (u32)NXF) {
      soff[lane] = incl - c;
      sbase[lane] = c ? atomicAdd(&W.cnt[W.wr_cnt * NXF + lane], c) : 0u;
    }
    if (lane == 31u) soff[NXF] = incl;
  }
  __syncthreads();
  if (alive) {
    const u32 q = soff[nfn] + rank;
    sperm[q] = (unsigned short)t;
    skey[q] = (unsigned char)nfn;
    sdst[q] = sbase[nfn] + rank;
  }
  __syncthreads();
  if (t < soff[NXF]) {
    const u32 src = sperm[t], kk = skey[t], g = sdst[t];
    // Written with an evict-last L2 policy: the next launch of this
    // population reads the records back.
    u64 pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    u32* dst = wave_field(W, W.wr_buf, kk, 0) + g;
#pragma unroll 4
    for (u32 f = 0; f < (u32)WRNG; ++f, dst += W.cap) st_keep(dst, srng[f * WB + src], pol);
#pragma unroll
    for (u32 f = 0; f < 6u; ++f, dst += W.cap) st_keep(dst, sfs[f * WB + src], pol);
  }
}
#endif  // WAVE

// ------------------------------------------------------- stage test kernels
// Xform pick of an explicit draw stream (chaos.wgsl:8343-8348).
extern "C" __global__ void pick_test_kernel(const unsigned short* pick_start, u32 count,
                                            const int* prev, const u32* draws, u32* out) {
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  u32 row = prev[i] >= 0 ? (u32)prev[i] : (u32)NXF;
  out[i] = pick_xform(pick_start, row, draws[i] & 16383u);
}

// Splat of an explicit point stream (x, y, colour, opacity) with the chaos
// kernel's scatter; colour mode 0, no direct colour.
extern "C" __global__ void __launch_bounds__(WPB)
splat_test_kernel(const __grid_constant__ ChaosArgs A, u32 n, const float4* pts) {
  __shared__ float4 pal[256];
  for (u32 i = threadIdx.x; i < 256u; i += blockDim.x) pal[i] = ((const float4*)A.palette)[i];
  __syncthreads();
  u32 i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 q = pts[i];
  u64 n_in = 0;
  splat(A, pal, make_float3(q.x, q.y, q.z), f2(q.x, q.y), q.w, 0, make_float3(0.0f, 0.0f, 0.0f), &n_in);
}

// Device seeding, state written back in the reference layout
// [cnt, a, b, c, mem[16], rsl[16]] (src/isaac.ts:194-229).
extern "C" __global__ void __launch_bounds__(WPB)
seed_test_kernel(u32 seed, u64 base, u32 n, u32* out) {
  __shared__ u32 st[36 * WPB];
  u32 t = threadIdx.x;
  u64 i = (u64)blockIdx.x * WPB + t;
  if (i >= n) return;
  Rng r{st + t, WPB};
  seed_walker(r, seed, base + i);
  for (int k = 0; k < 36; ++k) out[i * 36 + k] = r.f(k);
}
