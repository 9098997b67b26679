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

VDEV float3 mix3(float3 a, float3 b, float t) {
  return make_float3(wmix(a.x, b.x, t), wmix(a.y, b.y, t), wmix(a.z, b.z, t));
}

// Palette mix a*(1-t) + b*t with separately rounded products (no FMA), so
// the fixed-point deposit is bit-identical to the reference arithmetic.
VDEV float mix_rn(float a, float b, float t) {
  return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
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
            o.pv = f2(wmix(o.pv.x, ob.pv.x, tb), wmix(o.pv.y, ob.pv.y, tb));
            o.nz = wmix(o.nz, ob.nz, tb);
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
          float jx = (rand01(rng) - 0.5f) * amp;
          float jy = (rand01(rng) - 0.5f) * amp;
          wx[t] = pv.x + jx; wy[t] = pv.y + jy; wz[t] = nz;
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
