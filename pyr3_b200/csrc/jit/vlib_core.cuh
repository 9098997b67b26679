// pyr3-b200 variation library: core helpers shared by every variation.
//
// Compiled at run time by NVRTC (sm_100a) together with the generated chaos
// kernel for one genome structure.  No CUDA headers are included: NVRTC
// provides the math builtins.
//
// Numeric contract (the reference's WGSL semantics, chaos.wgsl:230-520):
//   * all iteration arithmetic is f32;
//   * trig of |a| > 1e6 is replaced by trig of a hash of the argument bits
//     (safe_sin/safe_cos, chaos.wgsl:356-372), tanh clamps its argument to
//     +-20 (chaos.wgsl:381-385);
//   * pow(x < 0, y) is NaN (GPU exp2(y*log2 x) semantics), float x % y is
//     x - y*trunc(x/y), round() is round-half-even, f32->int conversions
//     clamp (WGSL value conversion);
//   * RNG: one ISAAC (RANDSIZL=4) stream per walker, rand01 / rand_11 scale
//     the low 28 bits exactly as chaos.wgsl:319-331 / flam3.c:2625-2631.
#pragma once

typedef unsigned int u32;
typedef int i32;
typedef unsigned long long u64;

#define VDEV __device__ __forceinline__

// --------------------------------------------------- out-of-line libm
// CUDA's accurate transcendental paths are long; inlined at every call site
// of every variation they made one genome's specialised kernel larger than
// the SM instruction cache.  Each is compiled once here and called; the
// names below redirect the library (and the kernel) to these copies.  The
// values are the same functions' values.
#define OUTL __device__ __noinline__
OUTL float ol_sinf(float x) { return sinf(x); }
OUTL float ol_cosf(float x) { return cosf(x); }
OUTL float2 ol_sincos(float x) {
  float s, c;
  sincosf(x, &s, &c);
  return make_float2(s, c);
}
OUTL float ol_tanf(float x) { return tanf(x); }
OUTL float ol_expf(float x) { return expf(x); }
OUTL float ol_logf(float x) { return logf(x); }
OUTL float ol_log2f(float x) { return log2f(x); }
OUTL float ol_log10f(float x) { return log10f(x); }
OUTL float ol_powf(float x, float y) { return powf(x, y); }
OUTL float ol_atan2f(float y, float x) { return atan2f(y, x); }
OUTL float ol_atanf(float x) { return atanf(x); }
OUTL float ol_asinf(float x) { return asinf(x); }
OUTL float ol_acosf(float x) { return acosf(x); }
OUTL float ol_sinhf(float x) { return sinhf(x); }
OUTL float ol_coshf(float x) { return coshf(x); }
OUTL float ol_tanhf(float x) { return tanhf(x); }
OUTL float ol_asinhf(float x) { return asinhf(x); }
OUTL float ol_acoshf(float x) { return acoshf(x); }
OUTL float ol_atanhf(float x) { return atanhf(x); }
OUTL double ol_sin(double x) { return sin(x); }
#define sinf ol_sinf
#define cosf ol_cosf
#define tanf ol_tanf
#define expf ol_expf
#define logf ol_logf
#define log2f ol_log2f
#define log10f ol_log10f
#define powf ol_powf
#define atan2f ol_atan2f
#define atanf ol_atanf
#define asinf ol_asinf
#define acosf ol_acosf
#define sinhf ol_sinhf
#define coshf ol_coshf
#define tanhf ol_tanhf
#define asinhf ol_asinhf
#define acoshf ol_acoshf
#define atanhf ol_atanhf
#define sin ol_sin

#define P_PI 3.14159265358979323846f
#define P_TAU 6.28318530717958647692f
#define P_HALF_PI 1.57079632679489661923f
#define P_EPS 1e-10f
#define P_LN10 2.302585092994046f

// ----------------------------------------------------------------- float2
VDEV float2 f2(float x, float y) { return make_float2(x, y); }
VDEV float2 operator+(float2 a, float2 b) { return f2(a.x + b.x, a.y + b.y); }
VDEV float2 operator-(float2 a, float2 b) { return f2(a.x - b.x, a.y - b.y); }
VDEV float2 operator-(float2 a) { return f2(-a.x, -a.y); }
VDEV float2 operator*(float2 a, float s) { return f2(a.x * s, a.y * s); }
VDEV float2 operator*(float s, float2 a) { return f2(s * a.x, s * a.y); }
VDEV float2 operator*(float2 a, float2 b) { return f2(a.x * b.x, a.y * b.y); }
VDEV float2 operator/(float2 a, float s) { return f2(a.x / s, a.y / s); }
VDEV float2& operator+=(float2& a, float2 b) { a.x += b.x; a.y += b.y; return a; }
VDEV float dot2(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
VDEV float sq2(float2 a) { return a.x * a.x + a.y * a.y; }
VDEV float len2(float2 a) { return sqrtf(a.x * a.x + a.y * a.y); }
// Separately rounded products, for expressions whose outcome hinges on the
// last bit (a branch on a near-zero discriminant, a hash of a product, an
// angle of 1e5 rad): the compiler never fuses an __fmul_rn into an add, so
// these round exactly as the reference's f32 operations do.
VDEV float mul_rn(float a, float b) { return __fmul_rn(a, b); }
VDEV float dot_rn(float ax, float ay, float bx, float by) { return mul_rn(ax, bx) + mul_rn(ay, by); }
VDEV float len_rn(float x, float y) { return sqrtf(mul_rn(x, x) + mul_rn(y, y)); }

// ------------------------------------------------------- WGSL semantics
VDEV float wpow(float x, float y) {
  return x < 0.0f ? __int_as_float(0x7fffffff) : powf(x, y);
}
VDEV float wmod(float x, float y) { return x - y * truncf(x / y); }
VDEV float wfract(float x) { return x - floorf(x); }
VDEV float wround(float x) { return rintf(x); }
VDEV float wsign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
VDEV float wclamp(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
VDEV float wmix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
VDEV float wstep(float edge, float x) { return edge <= x ? 1.0f : 0.0f; }
VDEV float wsmooth(float lo, float hi, float x) {
  float t = wclamp((x - lo) / (hi - lo), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
VDEV i32 f2i(float v) {  // WGSL i32(f32): truncate, clamp, NaN -> 0
  if (!(v == v)) return 0;
  return v <= -2147483648.0f ? (i32)0x80000000 : (v >= 2147483520.0f ? 2147483520 : (i32)v);
}
VDEV u32 f2u(float v) {  // WGSL u32(f32)
  if (!(v > 0.0f)) return 0u;
  return v >= 4294967040.0f ? 4294967040u : (u32)v;
}
VDEV i32 imod(i32 a, i32 b) {  // WGSL i32 %: x % 0 = 0
  return b == 0 ? 0 : ((a == (i32)0x80000000 && b == -1) ? 0 : a % b);
}
VDEV i32 idiv(i32 a, i32 b) {  // WGSL i32 /: x / 0 = x
  return b == 0 ? a : ((a == (i32)0x80000000 && b == -1) ? a : a / b);
}

// ------------------------------------------------------------ safe trig
VDEV float hash01(u32 h) {
  h ^= h >> 17; h *= 0xed5ad4bbu;
  h ^= h >> 11; h *= 0xac4c1b51u;
  h ^= h >> 15;
  return (float)h * (1.0f / 4294967296.0f);
}
VDEV float safe_arg(float a) {  // |a| > 1e6: trig of a hash of the bits
  return fabsf(a) <= 1.0e6f ? a : hash01(__float_as_uint(a)) * P_TAU;
}
VDEV float ssin(float a) { return sinf(safe_arg(a)); }
VDEV float scos(float a) { return cosf(safe_arg(a)); }
VDEV void ssincos(float a, float* s, float* c) {
  float2 r = ol_sincos(safe_arg(a));
  *s = r.x;
  *c = r.y;
}
VDEV float stan(float a) { return ssin(a) / scos(a); }
VDEV float stanh(float a) { return tanhf(wclamp(a, -20.0f, 20.0f)); }
VDEV float2 polar2(float r, float ang) {  // (r cos a, r sin a) with safe trig
  float s, c;
  ssincos(ang, &s, &c);
  return f2(r * c, r * s);
}

// ------------------------------------------------------------ RNG state
// One ISAAC stream per walker, held in shared memory as a [36][W] array of
// u32 so that a warp touching 32 consecutive walkers hits 32 banks whatever
// field it reads: field 0 = cnt, 1..3 = a, b, c, 4..19 = mem, 20..35 = rsl.
// The wave kernel refills early (isaac_early_refill): it then keeps the
// unread results of the old block in fields 36..42 and their count in bits
// 8..15 of field 0, and irand serves those first.
struct Rng {
  u32* s;  // &state[0][walker]
  u32 W;   // walkers per block (stride between fields)
  VDEV u32& f(u32 k) const { return s[k * W]; }
};

// One ISAAC round (Jenkins' isaac() with RANDSIZL = 4), flam3 isaac.c,
// on the state at s (fields W words apart).  Out of line: it runs once per
// sixteen draws, and inlined at every draw site it dominated the code size.
OUTL void isaac_round_at(u32* s, u32 W) {
  u32 a = s[1 * W];
  u32 c = s[3 * W] + 1u;
  s[3 * W] = c;
  u32 b = s[2 * W] + c;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int m = i, m2 = (i + 8) & 15;
    u32 mixed;
    switch (i & 3) {
      case 0: mixed = a ^ (a << 13); break;
      case 1: mixed = a ^ (a >> 6); break;
      case 2: mixed = a ^ (a << 2); break;
      default: mixed = a ^ (a >> 16); break;
    }
    u32 x = s[(4 + m) * W];
    a = mixed + s[(4 + m2) * W];
    u32 y = s[(4 + ((x >> 2) & 15u)) * W] + a + b;
    s[(4 + m) * W] = y;
    b = s[(4 + ((y >> 6) & 15u)) * W] + x;
    s[(20 + m) * W] = b;
  }
  s[1 * W] = a;
  s[2 * W] = b;
}
VDEV void isaac_round(const Rng& r) { isaac_round_at(r.s, r.W); }

VDEV u32 irand(const Rng& r) {
  u32 cnt = r.f(0);
  if (cnt >= 256u) {  // results stashed by an early refill come first
    const u32 sc = (cnt >> 8) - 1u;
    r.f(0) = (sc << 8) | (cnt & 0xffu);
    return r.f(36 + sc);
  }
  if (cnt == 0u) {
    isaac_round(r);
    cnt = 15u;
  } else {
    cnt -= 1u;
  }
  r.f(0) = cnt;
  return r.f(20 + cnt);
}
VDEV float rand01(const Rng& r) {
  return (float)(irand(r) & 0x0fffffffu) * (1.0f / 268435455.0f);
}
VDEV float rand_11(const Rng& r) {
  return (float)((i32)(irand(r) & 0x0fffffffu) - 0x07ffffff) * (1.0f / 134217727.0f);
}

// ------------------------------------------------------ variation context
// Everything a variation may read besides its input point, weight and its
// ten parameters: the walker's RNG and the owning xform's affine
// coefficients (a0 = [a, b, c, weight], a1 = [d, e, f, nvars]).
struct Ctx {
  Rng rng;
  float4 a0, a1;
};

#define VAR(name) VDEV float2 var_##name(float2 p, float w, const float* __restrict__ P, Ctx& c)
#define RAND01() rand01(c.rng)
#define RAND11() rand_11(c.rng)
#define IRAND() irand(c.rng)

// --------------------------------------------------------------- complex
// z = (re, im).  Division / reciprocal floor |b|^2 at 0 (the reference's
// 1e-100 floor rounds to 0 in f32).
VDEV float2 cmul(float2 a, float2 b) { return f2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
VDEV float2 csqr(float2 z) { return f2(z.x * z.x - z.y * z.y, 2.0f * z.x * z.y); }
VDEV float2 cdiv(float2 a, float2 b) {
  float m2 = fmaxf(dot2(b, b), 0.0f);
  return f2((a.x * b.x + a.y * b.y) / m2, (a.y * b.x - a.x * b.y) / m2);
}
VDEV float2 crecip(float2 z) {
  float m2 = fmaxf(dot2(z, z), 0.0f);
  return f2(z.x / m2, -z.y / m2);
}
VDEV float2 csqrt(float2 z) {
  float rad = len2(z);
  float sb = z.y < 0.0f ? -1.0f : 1.0f;
  return f2(sqrtf(fmaxf(0.5f * (rad + z.x), 0.0f)), sb * sqrtf(fmaxf(0.5f * (rad - z.x), 0.0f)));
}
VDEV float2 clog(float2 z) {
  return f2(0.5f * logf(dot2(z, z) + 1e-20f), atan2f(z.y, z.x));
}
VDEV float2 cexp(float2 z) {
  float e = expf(wclamp(z.x, -20.0f, 20.0f));
  float s, co;
  ssincos(z.y, &s, &co);
  return f2(e * co, e * s);
}
VDEV float2 cpowc(float2 t, float2 p) { return cexp(cmul(p, clog(t))); }
VDEV float2 csin(float2 z) {
  float y = wclamp(z.y, -20.0f, 20.0f);
  float ep = expf(y), en = expf(-y);
  float ch = 0.5f * (ep + en), sh = 0.5f * (ep - en);
  return f2(ssin(z.x) * ch, scos(z.x) * sh);
}

// ----------------------------------------------------------------- colour
// hsv_to_rgb (chaos.wgsl:1662): v * mix(1, clamp(|fract(h + k)*6 - 3| - 1),
// s) with k = (1, 2/3, 1/3).
VDEV float3 hsv_rgb(float h, float s, float v) {
  const float k[3] = {1.0f, 2.0f / 3.0f, 1.0f / 3.0f};
  float o[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float q = fabsf(wfract(h + k[i]) * 6.0f - 3.0f);
    o[i] = v * wmix(1.0f, wclamp(q - 1.0f, 0.0f, 1.0f), s);
  }
  return make_float3(o[0], o[1], o[2]);
}
// hsl_to_rgb (chaos.wgsl:1696).
VDEV float3 hsl_rgb(float hh, float ss, float ll) {
  float h = wfract(hh), s = wclamp(ss, 0.0f, 1.0f), l = wclamp(ll, 0.0f, 1.0f);
  float cc = (1.0f - fabsf(2.0f * l - 1.0f)) * s;
  float h6 = h * 6.0f;
  float x = cc * (1.0f - fabsf((h6 - 2.0f * floorf(h6 * 0.5f)) - 1.0f));
  float m = l - cc * 0.5f;
  float r, g, b;
  if (h6 < 1.0f) { r = cc; g = x; b = 0.0f; }
  else if (h6 < 2.0f) { r = x; g = cc; b = 0.0f; }
  else if (h6 < 3.0f) { r = 0.0f; g = cc; b = x; }
  else if (h6 < 4.0f) { r = 0.0f; g = x; b = cc; }
  else if (h6 < 5.0f) { r = x; g = 0.0f; b = cc; }
  else { r = cc; g = 0.0f; b = x; }
  return make_float3(r + m, g + m, b + m);
}
#define DCV(name) VDEV float3 dc_##name(float2 p, const float* __restrict__ P)
