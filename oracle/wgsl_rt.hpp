// Runtime for the C++ that oracle/wgsl2cpp.py emits from the reference's WGSL
// shaders.  TEST INFRASTRUCTURE ONLY (the oracle), never part of the product.
//
// Implements WGSL value semantics on the host in f32: vector types and
// operators, the builtin functions the reference shaders call, the clamping
// float->int conversions, integer division/remainder rules (x/0 = x,
// x%0 = 0), masked shift counts and float `%` = e1 - e2*trunc(e1/e2).
// Transcendentals use the C library's f32 functions; pow() of a negative base
// is NaN, as GPU exp2(y*log2(x)) lowerings make it.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <type_traits>

namespace wg {

template <class T, int N> struct vec;
template <class T> struct vec<T, 2> {
  T x{}, y{};
  vec() = default;
  constexpr vec(T a, T b) : x(a), y(b) {}
  T &operator[](int i) { return i == 0 ? x : y; }
  const T &operator[](int i) const { return i == 0 ? x : y; }
};
template <class T> struct vec<T, 3> {
  T x{}, y{}, z{};
  vec() = default;
  constexpr vec(T a, T b, T c) : x(a), y(b), z(c) {}
  T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  const T &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class T> struct vec<T, 4> {
  T x{}, y{}, z{}, w{};
  vec() = default;
  constexpr vec(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
  T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  const T &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

template <class T> struct is_vec : std::false_type {};
template <class T, int N> struct is_vec<vec<T, N>> : std::true_type {};
template <class T> struct elem { using type = T; static constexpr int n = 1; };
template <class T, int N> struct elem<vec<T, N>> { using type = T; static constexpr int n = N; };

template <class T> inline T comp(const T &s, int) { return s; }
template <class T, int N> inline T comp(const vec<T, N> &v, int i) { return v[i]; }

// ---- scalar conversions with WGSL rules ----
template <class To, class From> inline To cvt(From v) {
  if constexpr (std::is_same_v<To, From>) {
    return v;
  } else if constexpr (std::is_same_v<To, bool>) {
    return v != From(0);
  } else if constexpr (std::is_floating_point_v<From> && std::is_integral_v<To>) {
    if (v != v) return To(0);
    const double lo = (double)std::numeric_limits<To>::min();
    // largest f32 below the integer type's max, as the WGSL spec clamps
    const double hi = std::is_same_v<To, int32_t> ? 2147483520.0 : 4294967040.0;
    double d = (double)v;
    if (d <= lo) return std::numeric_limits<To>::min();
    if (d >= hi) return (To)hi;
    return (To)d;
  } else if constexpr (std::is_same_v<From, bool>) {
    return v ? To(1) : To(0);
  } else if constexpr (std::is_integral_v<From> && std::is_integral_v<To>) {
    return (To)(std::make_unsigned_t<From>)v;  // bit reinterpretation / wrap
  } else {
    return (To)v;
  }
}

// ---- constructors: flatten scalars/vectors into components ----
template <class R> struct builder {
  using S = typename elem<R>::type;
  static constexpr int N = elem<R>::n;
  S c[4]{};
  int k = 0;
  template <class A> void push(const A &a) {
    if constexpr (is_vec<A>::value) {
      for (int i = 0; i < elem<A>::n; ++i) c[k++] = cvt<S>(a[i]);
    } else {
      c[k++] = cvt<S>(a);
    }
  }
};
template <class R, class... A> inline R make(const A &...a) {
  builder<R> b;
  (b.push(a), ...);
  if constexpr (!is_vec<R>::value) {
    return b.c[0];
  } else {
    using S = typename elem<R>::type;
    constexpr int N = elem<R>::n;
    if (b.k == 1) for (int i = 1; i < N; ++i) b.c[i] = b.c[0];  // splat
    R r;
    for (int i = 0; i < N; ++i) r[i] = b.c[i];
    (void)sizeof(S);
    return r;
  }
}
template <class R, class A> inline R conv(const A &a) {
  if constexpr (is_vec<R>::value && is_vec<A>::value) {
    R r;
    for (int i = 0; i < elem<R>::n; ++i) r[i] = cvt<typename elem<R>::type>(a[i]);
    return r;
  } else {
    return make<R>(a);
  }
}
template <class To, class From> inline To bitcast(const From &f) {
  if constexpr (sizeof(To) != sizeof(From) && std::is_same_v<From, double>) {
    // FP64 build of the shaders (oracle/build.py, f32 emitted as double):
    // a WGSL bitcast of an f32 reads the bits of the value rounded to f32.
    return bitcast<To>((float)f);
  } else if constexpr (sizeof(To) != sizeof(From) && std::is_same_v<To, double>) {
    return (double)bitcast<float>(f);
  } else {
    static_assert(sizeof(To) == sizeof(From), "bitcast size");
    To t;
    std::memcpy(&t, &f, sizeof t);
    return t;
  }
}

// ---- elementwise helpers ----
template <class A, class B> struct vres { using type = A; };
template <class T, int N> struct vres<T, vec<T, N>> { using type = vec<T, N>; };
template <class F, class A> inline auto map1(F f, const A &a) {
  if constexpr (is_vec<A>::value) {
    A r;
    for (int i = 0; i < elem<A>::n; ++i) r[i] = f(a[i]);
    return r;
  } else {
    return f(a);
  }
}
template <class F, class A, class B> inline auto map2(F f, const A &a, const B &b) {
  using R = typename vres<A, B>::type;
  if constexpr (is_vec<R>::value) {
    R r;
    for (int i = 0; i < elem<R>::n; ++i) r[i] = f(comp(a, i), comp(b, i));
    return r;
  } else {
    return f(a, b);
  }
}
template <class F, class A, class B, class C> inline auto map3(F f, const A &a, const B &b, const C &c) {
  using R = typename vres<typename vres<A, B>::type, C>::type;
  if constexpr (is_vec<R>::value) {
    R r;
    for (int i = 0; i < elem<R>::n; ++i) r[i] = f(comp(a, i), comp(b, i), comp(c, i));
    return r;
  } else {
    return f(a, b, c);
  }
}

// ---- arithmetic operators on vectors ----
#define WG_BINOP(OP)                                                                        \
  template <class T, int N> inline vec<T, N> operator OP(const vec<T, N> &a, const vec<T, N> &b) { \
    vec<T, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] OP b[i]; return r; }              \
  template <class T, int N> inline vec<T, N> operator OP(const vec<T, N> &a, T b) {          \
    vec<T, N> r; for (int i = 0; i < N; ++i) r[i] = a[i] OP b; return r; }                 \
  template <class T, int N> inline vec<T, N> operator OP(T a, const vec<T, N> &b) {          \
    vec<T, N> r; for (int i = 0; i < N; ++i) r[i] = a OP b[i]; return r; }                 \
  template <class T, int N, class B> inline vec<T, N> &operator OP##=(vec<T, N> &a, const B &b) { \
    a = a OP b; return a; }
WG_BINOP(+)
WG_BINOP(-)
WG_BINOP(*)
WG_BINOP(&)
WG_BINOP(|)
WG_BINOP(^)
#undef WG_BINOP
template <class T, int N> inline vec<T, N> operator-(const vec<T, N> &a) {
  vec<T, N> r; for (int i = 0; i < N; ++i) r[i] = -a[i]; return r;
}
template <class T, int N> inline vec<T, N> operator~(const vec<T, N> &a) {
  vec<T, N> r; for (int i = 0; i < N; ++i) r[i] = ~a[i]; return r;
}
template <int N> inline vec<bool, N> operator!(const vec<bool, N> &a) {
  vec<bool, N> r; for (int i = 0; i < N; ++i) r[i] = !a[i]; return r;
}
#define WG_CMP(NAME, OP)                                                                        \
  template <class A, class B> inline auto NAME(const A &a, const B &b) {                        \
    using R = typename vres<A, B>::type;                                                        \
    if constexpr (is_vec<R>::value) {                                                           \
      vec<bool, elem<R>::n> r; for (int i = 0; i < elem<R>::n; ++i) r[i] = comp(a, i) OP comp(b, i); \
      return r;                                                                                 \
    } else { return a OP b; } }
WG_CMP(eq, ==)
WG_CMP(ne, !=)
WG_CMP(lt, <)
WG_CMP(le, <=)
WG_CMP(gt, >)
WG_CMP(ge, >=)
#undef WG_CMP

// division and remainder with WGSL integer rules
template <class T> inline T div_s(T a, T b) {
  if constexpr (std::is_floating_point_v<T>) {
    return a / b;
  } else if constexpr (std::is_signed_v<T>) {
    if (b == 0) return a;
    if (a == std::numeric_limits<T>::min() && b == -1) return a;
    return a / b;
  } else {
    return b == 0 ? a : a / b;
  }
}
template <class T> inline T mod_s(T a, T b) {
  if constexpr (std::is_floating_point_v<T>) {
    return a - b * std::trunc(a / b);
  } else if constexpr (std::is_signed_v<T>) {
    if (b == 0) return 0;
    if (a == std::numeric_limits<T>::min() && b == -1) return 0;
    return a % b;
  } else {
    return b == 0 ? 0 : a % b;
  }
}
template <class A, class B> inline auto div(const A &a, const B &b) {
  return map2([](auto x, auto y) { return div_s<decltype(x)>(x, y); }, a, b);
}
template <class A, class B> inline auto mod(const A &a, const B &b) {
  return map2([](auto x, auto y) { return mod_s<decltype(x)>(x, y); }, a, b);
}
template <class A, class B> inline auto shl(const A &a, const B &b) {
  return map2([](auto x, auto y) {
    using T = decltype(x);
    return (T)((std::make_unsigned_t<T>)x << ((uint32_t)y & (sizeof(T) * 8 - 1)));
  }, a, b);
}
template <class A, class B> inline auto shr(const A &a, const B &b) {
  return map2([](auto x, auto y) {
    using T = decltype(x);
    return (T)(x >> ((uint32_t)y & (sizeof(T) * 8 - 1)));
  }, a, b);
}

// ---- builtins ----
template <class T> inline T fsel(float f, double d) { return std::is_same_v<T, float> ? (T)f : (T)d; }
#define WG_F1(NAME, EXPR)                                                  \
  template <class A> inline auto NAME(const A &a) {                        \
    return map1([](auto x) { using T = decltype(x); (void)sizeof(T); return EXPR; }, a); }
// sin / cos / tan of an f32 are the correctly rounded f32 value (evaluated
// in f64, rounded once).  WGSL leaves their accuracy to the implementation;
// this fixes one canonical answer, and the hash-style variations
// (fract(sin(.) * 43758.5453)) depend on every bit of it.
WG_F1(sin, (T)std::sin((double)x))
WG_F1(cos, (T)std::cos((double)x))
WG_F1(tan, (T)std::tan((double)x))
WG_F1(asin, (T)std::asin(x))
WG_F1(acos, (T)std::acos(x))
WG_F1(atan, (T)std::atan(x))
WG_F1(sinh, (T)std::sinh(x))
WG_F1(cosh, (T)std::cosh(x))
WG_F1(tanh, (T)std::tanh(x))
WG_F1(asinh, (T)std::asinh(x))
WG_F1(acosh, (T)std::acosh(x))
WG_F1(atanh, (T)std::atanh(x))
WG_F1(exp, (T)std::exp(x))
WG_F1(exp2, (T)std::exp2(x))
WG_F1(log, (T)std::log(x))
WG_F1(log2, (T)std::log2(x))
WG_F1(sqrt, (T)std::sqrt(x))
WG_F1(inverseSqrt, (T)(T(1) / std::sqrt(x)))
WG_F1(floor, (T)std::floor(x))
WG_F1(ceil, (T)std::ceil(x))
WG_F1(trunc, (T)std::trunc(x))
WG_F1(round, (T)std::nearbyint(x))
WG_F1(fract, (T)(x - std::floor(x)))
WG_F1(saturate, (T)std::fmin(std::fmax(x, T(0)), T(1)))
WG_F1(degrees, (T)(x * (T)57.295779513082320876798))
WG_F1(radians, (T)(x * (T)0.017453292519943295769237))
WG_F1(sign, (T)((x > T(0)) ? T(1) : ((x < T(0)) ? T(-1) : T(0))))
#undef WG_F1
template <class A> inline auto abs(const A &a) {
  return map1([](auto x) {
    using T = decltype(x);
    if constexpr (std::is_floating_point_v<T>) return (T)std::fabs(x);
    else if constexpr (std::is_signed_v<T>) return x == std::numeric_limits<T>::min() ? x : (x < 0 ? -x : x);
    else return x;
  }, a);
}
template <class A, class B> inline auto atan2(const A &a, const B &b) {
  return map2([](auto y, auto x) { using T = decltype(y); return (T)std::atan2(y, (T)x); }, a, b);
}
template <class A, class B> inline auto pow(const A &a, const B &b) {
  return map2([](auto x, auto y) {
    using T = decltype(x);
    if (x < T(0)) return std::numeric_limits<T>::quiet_NaN();
    return (T)std::pow(x, (T)y);
  }, a, b);
}
template <class A, class B> inline auto min(const A &a, const B &b) {
  return map2([](auto x, auto y) {
    using T = decltype(x);
    if constexpr (std::is_floating_point_v<T>) return (T)std::fmin(x, (T)y);
    else return x < (T)y ? x : (T)y;
  }, a, b);
}
template <class A, class B> inline auto max(const A &a, const B &b) {
  return map2([](auto x, auto y) {
    using T = decltype(x);
    if constexpr (std::is_floating_point_v<T>) return (T)std::fmax(x, (T)y);
    else return x > (T)y ? x : (T)y;
  }, a, b);
}
template <class A, class B, class C> inline auto clamp(const A &e, const B &lo, const C &hi) {
  return min(max(e, lo), hi);
}
template <class A, class B> inline auto step(const A &edge, const B &x) {
  return map2([](auto e, auto v) { using T = decltype(v); return (T)(e <= v ? T(1) : T(0)); }, edge, x);
}
template <class A, class B, class C> inline auto mix(const A &a, const B &b, const C &t) {
  return map3([](auto x, auto y, auto s) { using T = decltype(x); return (T)(x * (T(1) - s) + y * s); }, a, b, t);
}
template <class A, class B, class C> inline auto smoothstep(const A &lo, const B &hi, const C &x) {
  return map3([](auto l, auto h, auto v) {
    using T = decltype(v);
    T t = (T)std::fmin(std::fmax((v - l) / (h - l), T(0)), T(1));
    return (T)(t * t * (T(3) - T(2) * t));
  }, lo, hi, x);
}
template <class A, class B, class C> inline auto fma(const A &a, const B &b, const C &c) {
  return map3([](auto x, auto y, auto z) { using T = decltype(x); return (T)std::fma(x, y, z); }, a, b, c);
}
template <class T, int N> inline T dot(const vec<T, N> &a, const vec<T, N> &b) {
  T s = T(0);
  for (int i = 0; i < N; ++i) s = s + a[i] * b[i];
  return s;
}
template <class T> inline T length(const T &a) { return (T)std::fabs(a); }
template <class T, int N> inline T length(const vec<T, N> &a) { return (T)std::sqrt(dot(a, a)); }
template <class A> inline auto distance(const A &a, const A &b) { return length(a - b); }
template <class T, int N> inline vec<T, N> normalize(const vec<T, N> &a) {
  T l = length(a);
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r[i] = a[i] / l;
  return r;
}
template <class T> inline vec<T, 3> cross(const vec<T, 3> &a, const vec<T, 3> &b) {
  return vec<T, 3>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template <class T, int N> inline vec<T, N> reflect(const vec<T, N> &e1, const vec<T, N> &e2) {
  return e1 - e2 * (T(2) * dot(e2, e1));
}
template <class A, class B> inline A select(const A &f, const A &t, const B &c) {
  if constexpr (is_vec<B>::value) {
    A r;
    for (int i = 0; i < elem<A>::n; ++i) r[i] = c[i] ? t[i] : f[i];
    return r;
  } else {
    return c ? t : f;
  }
}
inline bool any(bool b) { return b; }
inline bool all(bool b) { return b; }
template <int N> inline bool any(const vec<bool, N> &v) {
  for (int i = 0; i < N; ++i) if (v[i]) return true;
  return false;
}
template <int N> inline bool all(const vec<bool, N> &v) {
  for (int i = 0; i < N; ++i) if (!v[i]) return false;
  return true;
}
template <class A> inline auto countOneBits(const A &a) {
  return map1([](auto x) { using T = decltype(x); return (T)__builtin_popcount((uint32_t)x); }, a);
}
template <class A> inline auto reverseBits(const A &a) {
  return map1([](auto x) {
    using T = decltype(x);
    uint32_t v = (uint32_t)x, r = 0;
    for (int i = 0; i < 32; ++i) { r = (r << 1) | (v & 1u); v >>= 1; }
    return (T)r;
  }, a);
}
template <class T, int... I, int N> inline vec<T, sizeof...(I)> swz(const vec<T, N> &v) {
  return vec<T, sizeof...(I)>(v[I]...);
}

// ---- atomics (shared host memory; GCC __atomic builtins) ----
struct atomic_cmpxchg_u32 {
  uint32_t old_value;
  bool exchanged;
};
inline uint32_t atomicLoad(uint32_t *p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline void atomicStore(uint32_t *p, uint32_t v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
inline uint32_t atomicAdd(uint32_t *p, uint32_t v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
inline uint32_t atomicMax(uint32_t *p, uint32_t v) {
  uint32_t o = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (v > o && !__atomic_compare_exchange_n(p, &o, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
  return o;
}
inline atomic_cmpxchg_u32 atomicCompareExchangeWeak(uint32_t *p, uint32_t cmp, uint32_t v) {
  uint32_t expected = cmp;
  bool ok = __atomic_compare_exchange_n(p, &expected, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
  return {expected, ok};
}

}  // namespace wg

using vec2f = wg::vec<float, 2>;
using vec3f = wg::vec<float, 3>;
using vec4f = wg::vec<float, 4>;
using vec2i = wg::vec<int32_t, 2>;
using vec3i = wg::vec<int32_t, 3>;
using vec4i = wg::vec<int32_t, 4>;
using vec2u = wg::vec<uint32_t, 2>;
using vec3u = wg::vec<uint32_t, 3>;
using vec4u = wg::vec<uint32_t, 4>;
using vec2b = wg::vec<bool, 2>;
using vec3b = wg::vec<bool, 3>;
using vec4b = wg::vec<bool, 4>;
