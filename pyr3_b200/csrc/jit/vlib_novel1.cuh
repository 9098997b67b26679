// pyr3-b200 variation library, part 6: indices 223..257 (complex_gamma ..
// cantor_stairs), restated from the reference's src/shaders/chaos.wgsl
// lines 5532-6013.
#pragma once

VAR(complex_gamma) {  // P = scale; Lanczos (g = 7, 9 terms) with reflection
  const float g = 7.0f, s2pi = 2.5066282746310002f;
  const float cf[8] = {676.5203681218851f,    -1259.1392167224028f,   771.32342877765313f,
                       -176.61502916214059f,  12.507343278686905f,    -0.13857109526572012f,
                       9.9843695780195716e-6f, 1.5056327351493116e-7f};
  float2 z = p;
  bool refl = z.x < 0.5f;
  if (refl) z = f2(1.0f - z.x, -z.y);
  float2 x = z - f2(1.0f, 0.0f);
  float2 A = f2(0.99999999999980993f, 0.0f);
#pragma unroll
  for (int k = 0; k < 8; ++k) A = A + cdiv(f2(cf[k], 0.0f), x + f2((float)(k + 1), 0.0f));
  float2 t = x + f2(g + 0.5f, 0.0f);
  float2 res = s2pi * cmul(cpowc(t, x + f2(0.5f, 0.0f)), cmul(cexp(-t), A));
  if (refl) res = cdiv(cdiv(f2(3.14159265f, 0.0f), csin(3.14159265f * p)), res);
  return (w * P[0]) * res;
}
VAR(lambert_w) {  // P = iterations; Halley iteration for W(z)
  const i32 it = min(max(f2i(P[0] + 0.5f), 1), 4);
  float2 wn;
  if (len2(p) < 2.0f) {
    wn = clog(f2(1.0f, 0.0f) + p);
  } else {
    float2 lz = clog(p);
    wn = lz - clog(lz);
  }
  for (i32 i = 0; i < 4 && i < it; ++i) {
    float2 ew = cexp(wn);
    float2 f = cmul(wn, ew) - p;
    float2 wp1 = wn + f2(1.0f, 0.0f), wp2 = wn + f2(2.0f, 0.0f);
    float2 t = 2.0f * wp1;
    if (dot2(t, t) < 1.0e-20f) break;
    float2 den = cmul(ew, wp1) - cdiv(cmul(wp2, f), t);
    if (dot2(den, den) < 1.0e-20f) break;
    wn = wn - cdiv(f, den);
  }
  return w * wn;
}
VAR(mercator) {
  float lat = wclamp(p.y, -1.5f, 1.5f);
  return w * f2(p.x, logf(fabsf(stan(0.78539816f + lat * 0.5f)) + 1e-6f));
}
VAR(lambert) {
  float cy = scos(p.y);
  float k = sqrtf(2.0f / (1.0f + cy * scos(p.x) + 1e-6f));
  return w * f2(k * cy * ssin(p.x), k * ssin(p.y));
}
VAR(mollweide) {
  float t = p.y, tgt = 3.14159265f * ssin(p.y);
  for (int i = 0; i < 4; ++i) {
    float s2, c2;
    ssincos(2.0f * t, &s2, &c2);
    float df = 2.0f + 2.0f * c2;
    if (fabsf(df) < 1e-6f) break;
    t -= (2.0f * t + s2 - tgt) / df;
  }
  return w * f2(0.9003163f * p.x * scos(t), 1.4142135f * ssin(t));
}
VAR(hammer) {
  float cy = scos(p.y);
  float z = sqrtf(1.0f + cy * scos(p.x * 0.5f) + 1e-6f);
  return w * f2((2.828427f * cy * ssin(p.x * 0.5f)) / z, (1.4142135f * ssin(p.y)) / z);
}
VAR(stereographic) {
  float cy = scos(p.y);
  float k = 2.0f / (1.0f + cy * scos(p.x) + 1e-6f);
  return w * f2(k * cy * ssin(p.x), k * ssin(p.y));
}
VAR(standard_map) {  // P = k
  float xp = p.x + P[0] * ssin(p.y);
  return w * f2(xp, p.y + xp);
}
VAR(de_jong) {  // P = a, b, c, d
  return w * f2(ssin(P[0] * p.y) - scos(P[1] * p.x), ssin(P[2] * p.x) - scos(P[3] * p.y));
}
VAR(ikeda) {  // P = u
  float st, ct;
  ssincos(0.4f - 6.0f / (1.0f + p.x * p.x + p.y * p.y), &st, &ct);
  return w * f2(1.0f + P[0] * (p.x * ct - p.y * st), P[0] * (p.x * st + p.y * ct));
}
VDEV float box_fold1(float v, float lim) {
  return v > lim ? 2.0f * lim - v : (v < -lim ? -2.0f * lim - v : v);
}
VAR(box_fold) { return w * f2(box_fold1(p.x, P[0]), box_fold1(p.y, P[0])); }  // P = limit
VDEV float sphere_fold_scale(float r2, float rmin, float rmax) {
  float n2 = rmin * rmin, x2 = rmax * rmax;
  if (r2 < n2) return x2 / n2;
  if (r2 < x2) return x2 / fmaxf(r2, 1e-6f);
  return 1.0f;
}
VAR(sphere_fold) {  // P = rmin, rmax
  float s = sphere_fold_scale(p.x * p.x + p.y * p.y, P[0], P[1]);
  return w * f2(p.x * s, p.y * s);
}
VAR(mandelbox_step) {  // P = scale, rmin, rmax, cx, cy
  float x = box_fold1(p.x, 1.0f), y = box_fold1(p.y, 1.0f);
  float s = sphere_fold_scale(x * x + y * y, P[1], P[2]);
  return w * f2(x * s * P[0] + P[3], y * s * P[0] + P[4]);
}
VAR(kifs_fold) {  // P = n, offset
  float r = len2(p);
  if (r < 1e-6f) return f2(0.0f, 0.0f);
  float a = atan2f(p.y, p.x) - P[1];
  float th = 6.283185307179586f / fmaxf(1.0f, fabsf(P[0]));
  a -= th * floorf(a / th);
  if (a > th * 0.5f) a = th - a;
  return w * polar2(r, a + P[1]);
}
VAR(arnold_cat) {
  float xp = p.x * 2.0f + p.y, yp = p.x + p.y;
  return w * f2(wfract(xp + 0.5f) - 0.5f, wfract(yp + 0.5f) - 0.5f);
}
VAR(bakers_map) {
  float x = wfract(p.x + 0.5f), y = wfract(p.y + 0.5f);
  float xp = x < 0.5f ? 2.0f * x : 2.0f * x - 1.0f;
  float yp = x < 0.5f ? y * 0.5f : y * 0.5f + 0.5f;
  return w * f2(xp - 0.5f, yp - 0.5f);
}
VAR(tent_map) {
  float x = wfract(p.x + 0.5f), y = wfract(p.y + 0.5f);
  return w * f2((1.0f - fabsf(1.0f - 2.0f * x)) - 0.5f, (1.0f - fabsf(1.0f - 2.0f * y)) - 0.5f);
}
VAR(logistic_map) {  // P = r
  float x = wfract(p.x + 0.5f), y = wfract(p.y + 0.5f);
  return w * f2(P[0] * x * (1.0f - x) - 0.5f, P[0] * y * (1.0f - y) - 0.5f);
}
VAR(superellipse) {  // P = a, b, n
  float th = atan2f(p.y, p.x);
  float sa = fmaxf(fabsf(P[0]), 1e-4f), sb = fmaxf(fabsf(P[1]), 1e-4f), sn = fmaxf(P[2], 0.01f);
  float s, co;
  ssincos(th, &s, &co);
  float c0 = fabsf(co / sa), s0 = fabsf(s / sb);
  float r = wpow(fmaxf(wpow(c0, sn) + wpow(s0, sn), 1e-6f), -1.0f / sn);
  return w * f2(r * co, r * s);
}
VAR(limacon) {  // P = a, b
  float th = atan2f(p.y, p.x);
  float s, co;
  ssincos(th, &s, &co);
  float r = P[1] + P[0] * co;
  return w * f2(r * co, r * s);
}
VAR(epicycloid) {  // P = k
  float t = atan2f(p.y, p.x), k1 = P[0] + 1.0f;
  float s, co;
  ssincos(t, &s, &co);
  return w * f2(k1 * co - scos(k1 * t), k1 * s - ssin(k1 * t));
}
VAR(catenary) {  // P = a
  float sa = fmaxf(fabsf(P[0]), 1e-4f) * wsign(P[0] + 1e-8f);
  return w * f2(p.x, sa * coshf(p.x / sa));
}
VAR(tractrix) { return w * f2(p.x - stanh(p.x), 1.0f / coshf(p.x)); }
VAR(tinkerbell) {  // P = a, b, c, d
  return w * f2(p.x * p.x - p.y * p.y + P[0] * p.x + P[1] * p.y, 2.0f * p.x * p.y + P[2] * p.x + P[3] * p.y);
}
VAR(duffing) {  // P = h, delta, gamma, omega
  float xp = p.x + P[0] * p.y;
  float yp = p.y + P[0] * (p.x - p.x * p.x * p.x - P[1] * p.y + P[2] * scos(P[3] * p.x));
  return w * f2(xp, yp);
}
VAR(vanderpol) {  // P = h, mu
  return w * f2(p.x + P[0] * p.y, p.y + P[0] * (P[1] * (1.0f - p.x * p.x) * p.y - p.x));
}
VAR(rossler) {  // P = h, a
  float z = len2(p);
  return w * f2(p.x + P[0] * (-p.y - z), p.y + P[0] * (p.x + P[1] * p.y));
}
VAR(droste) {  // P = s
  float r = fmaxf(len2(p), 1e-6f), th = atan2f(p.y, p.x);
  float k = logf(fmaxf(P[0], 1e-4f)) / 6.283185307179586f;
  float lr = logf(r);
  float2 q = polar2(expf(lr - k * th), th + k * lr);
  return w * q;
}
VAR(logspiral) {  // P = a, k
  float th = atan2f(p.y, p.x);
  return w * polar2(P[0] * expf(P[1] * th), th);
}
VDEV float spiral_theta(float2 p) {
  float t = atan2f(p.y, p.x);
  return fmaxf(t < 0.0f ? t + 6.283185307179586f : t, 1e-6f);
}
VAR(fermat_spiral) {  // P = a
  float th = spiral_theta(p);
  return w * polar2(P[0] * sqrtf(th), th);
}
VAR(lituus) {  // P = a
  float th = spiral_theta(p);
  return w * polar2(P[0] / sqrtf(th), th);
}
VAR(hyperbolic_spiral) {  // P = a
  float th = spiral_theta(p);
  return w * polar2(P[0] / th, th);
}
VAR(weierstrass) {  // P = a, b, terms, amp
  float wx = 0.0f, wy = 0.0f, ap = 1.0f, bp = 1.0f;
  u32 n = f2u(wclamp(P[2], 1.0f, 16.0f));
  for (u32 i = 0; i < n; ++i) {
    wx += ap * scos(bp * 3.1415926535f * p.x);
    wy += ap * scos(bp * 3.1415926535f * p.y);
    ap *= P[0];
    bp *= P[1];
  }
  return w * f2(p.x + P[3] * wx, p.y + P[3] * wy);
}
VAR(takagi) {  // P = terms, amp
  float tx = 0.0f, ty = 0.0f, k = 1.0f;
  u32 n = f2u(wclamp(P[0], 1.0f, 16.0f));
  for (u32 i = 0; i < n; ++i) {
    float xs = k * p.x, ys = k * p.y;
    tx += fabsf(xs - floorf(xs + 0.5f)) / k;
    ty += fabsf(ys - floorf(ys + 0.5f)) / k;
    k *= 2.0f;
  }
  return w * f2(p.x + P[1] * tx, p.y + P[1] * ty);
}
VAR(cantor_stairs) {  // P = terms, amp
  float cx = p.x, cy = p.y;
  u32 n = f2u(wclamp(P[0], 1.0f, 8.0f));
  for (u32 i = 0; i < n; ++i) {
    cx = (cx + ssin(cx * 6.2831853f)) * 0.5f;
    cy = (cy + ssin(cy * 6.2831853f)) * 0.5f;
  }
  return w * f2(p.x + P[1] * cx, p.y + P[1] * cy);
}
