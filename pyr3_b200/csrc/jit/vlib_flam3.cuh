// pyr3-b200 variation library, part 1: the flam3 family, indices 0..98
// (src/variations.ts V map; kernels restated from src/shaders/chaos.wgsl
// lines 524-1660).  Angle conventions follow flam3's precalc flags:
// "xy" variations use atan2(x, y), "yx" variations atan2(y, x), and the
// "angles" family uses sin = x/r, cos = y/r (chaos.wgsl:12-47).
#pragma once

VAR(linear) { return p * w; }
VAR(sinusoidal) { return f2(w * ssin(p.x), w * ssin(p.y)); }
VAR(spherical) { return p * (w / (sq2(p) + P_EPS)); }
VAR(swirl) {
  float r2 = sq2(p), s, co;
  ssincos(r2, &s, &co);
  return f2(w * (s * p.x - co * p.y), w * (co * p.x + s * p.y));
}
VAR(horseshoe) {
  float k = w / (len2(p) + P_EPS);
  return f2(k * ((p.x - p.y) * (p.x + p.y)), k * (2.0f * p.x * p.y));
}
VAR(polar) { return f2(w * (atan2f(p.x, p.y) / P_PI), w * (len2(p) - 1.0f)); }
VAR(handkerchief) {
  float a = atan2f(p.x, p.y), r = len2(p), k = w * r;
  return f2(k * ssin(a + r), k * scos(a - r));
}
VAR(heart) {
  float a = atan2f(p.x, p.y), r = len2(p), k = w * r, s, co;
  ssincos(a * r, &s, &co);
  return f2(k * s, k * -co);
}
VAR(disc) {
  float k = w * (atan2f(p.x, p.y) / P_PI), s, co;
  ssincos(P_PI * len2(p), &s, &co);
  return f2(k * s, k * co);
}
VAR(spiral) {
  float r = len2(p) + P_EPS, s, co;
  ssincos(r, &s, &co);
  float k = w / r;
  return f2(k * (p.y / r + s), k * (p.x / r - co));
}
VAR(hyperbolic) {
  float r = len2(p) + P_EPS;
  return f2(w * ((p.x / r) / r), w * (r * (p.y / r)));
}
VAR(diamond) {
  float r = len2(p) + P_EPS, s, co;
  ssincos(len2(p), &s, &co);
  return f2(w * ((p.x / r) * co), w * ((p.y / r) * s));
}
VAR(ex) {
  float a = atan2f(p.x, p.y), r = len2(p);
  float n0 = ssin(a + r), n1 = scos(a - r);
  float m0 = n0 * n0 * n0, m1 = n1 * n1 * n1, k = w * r;
  return f2(k * (m0 + m1), k * (m0 - m1));
}
VAR(julia) {
  float th = atan2f(p.x, p.y) * 0.5f + ((IRAND() & 1u) == 1u ? P_PI : 0.0f);
  return polar2(w * sqrtf(len2(p)), th);
}
VAR(julian) {  // P = power, dist
  float r = len2(p), ph = atan2f(p.y, p.x);
  float n = floorf(RAND01() * fabsf(P[0]));
  return polar2(w * wpow(r, P[1] / P[0]), (ph + P_TAU * n) / P[0]);
}
VAR(bent) { return f2(w * (p.x < 0.0f ? p.x * 2.0f : p.x), w * (p.y < 0.0f ? p.y * 0.5f : p.y)); }
VAR(waves) {
  const float b = c.a0.y, cc = c.a0.z, e = c.a1.y, f = c.a1.z;
  return f2(w * (p.x + b * ssin(p.y / (cc * cc + P_EPS))), w * (p.y + e * ssin(p.x / (f * f + P_EPS))));
}
VAR(fisheye) {
  float k = w * (2.0f / (len2(p) + 1.0f));
  return f2(k * p.y, k * p.x);
}
VAR(popcorn) {
  return f2(w * (p.x + c.a0.z * ssin(stan(3.0f * p.y))), w * (p.y + c.a1.z * ssin(stan(3.0f * p.x))));
}
VAR(eyefish) { return p * (w * (2.0f / (len2(p) + 1.0f))); }
VAR(bubble) { return p * (w / (0.25f * sq2(p) + 1.0f)); }
VAR(cylinder) { return f2(w * ssin(p.x), w * p.y); }
VAR(disc2) {  // P = rot, twist
  const float rot = P[0], tw = P[1];
  float cosadd = scos(tw) - 1.0f, sinadd = ssin(tw);
  if (tw > P_TAU) {
    float k = 1.0f + tw - P_TAU;
    cosadd *= k; sinadd *= k;
  } else if (tw < -P_TAU) {
    float k = 1.0f + tw + P_TAU;
    cosadd *= k; sinadd *= k;
  }
  float s, co;
  ssincos((rot * P_PI) * (p.x + p.y), &s, &co);
  float r = (w * atan2f(p.x, p.y)) / P_PI;
  return f2((s + cosadd) * r, (co + sinadd) * r);
}
VAR(pdj) {  // P = a, b, c, d
  return f2(w * (ssin(P[0] * p.y) - scos(P[1] * p.x)), w * (ssin(P[2] * p.x) - scos(P[3] * p.y)));
}
VAR(exponential) { return polar2(w * expf(p.x - 1.0f), P_PI * p.y); }
VAR(power) {
  float r = len2(p) + P_EPS, sa = p.x / r, ca = p.y / r;
  float k = w * wpow(r, sa);
  return f2(k * ca, k * sa);
}
VAR(cosine) {
  float s, co;
  ssincos(p.x * P_PI, &s, &co);
  return f2(w * (co * coshf(p.y)), w * (-s * sinhf(p.y)));
}
VAR(tangent) { return f2(w * (ssin(p.x) / scos(p.y)), w * stan(p.y)); }
VAR(secant2) {
  float cr = scos(w * len2(p)), icr = 1.0f / cr;
  return f2(w * p.x, cr < 0.0f ? w * (icr + 1.0f) : w * (icr - 1.0f));
}
VAR(cross) {
  float s = p.x * p.x - p.y * p.y;
  return p * (w * sqrtf(1.0f / (s * s + P_EPS)));
}
VAR(rings) {
  float cc = c.a0.z, r0 = len2(p), re = r0 + P_EPS;
  float dx = cc * cc + P_EPS;
  float r = w * ((wmod(r0 + dx, 2.0f * dx) - dx) + r0 * (1.0f - dx));
  return f2(r * (p.y / re), r * (p.x / re));
}
VAR(fan) {
  float dx = P_PI * (c.a0.z * c.a0.z + P_EPS), dy = c.a1.z, dx2 = 0.5f * dx;
  float ph = atan2f(p.x, p.y), r = w * len2(p);
  float t = (ph + dy) - dx * truncf((ph + dy) / dx);
  return polar2(r, t > dx2 ? ph - dx2 : ph + dx2);
}
VAR(rings2) {  // P = val
  float r0 = len2(p), re = r0 + P_EPS, dx = P[0] * P[0] + P_EPS;
  float r = r0 - 2.0f * dx * truncf((r0 + dx) / (2.0f * dx)) + r0 * (1.0f - dx);
  float k = w * r;
  return f2(k * (p.x / re), k * (p.y / re));
}
VAR(fan2) {  // P = x, y
  float ph = atan2f(p.x, p.y), r = w * len2(p);
  float dy = P[1], dx = P_PI * (P[0] * P[0] + P_EPS), dx2 = 0.5f * dx;
  float t = ph + dy - dx * truncf((ph + dy) / dx);
  float a = t > dx2 ? ph - dx2 : ph + dx2, s, co;
  ssincos(a, &s, &co);
  return f2(r * s, r * co);
}
VAR(perspective) {  // P = angle, dist
  float ang = P[0] * (P_PI * 0.5f), vs = ssin(ang), vfc = P[1] * scos(ang);
  float t = 1.0f / (P[1] - p.y * vs);
  return f2(w * (P[1] * p.x * t), w * (vfc * p.y * t));
}
VAR(bipolar) {  // P = shift
  const float hp = P_PI * 0.5f, two_pi = 2.0f / P_PI;
  float x2y2 = sq2(p), t = x2y2 + 1.0f, x2 = 2.0f * p.x;
  float y = 0.5f * atan2f(2.0f * p.y, x2y2 - 1.0f) + (-hp * P[0]);
  if (y > hp) y = -hp + wmod(y + hp, P_PI);
  else if (y < -hp) y = hp - wmod(hp - y, P_PI);
  return f2(w * 0.25f * two_pi * logf((t + x2) / (t - x2)), w * two_pi * y);
}
VAR(curl) {  // P = c1, c2
  float re = 1.0f + P[0] * p.x + P[1] * (p.x * p.x - p.y * p.y);
  float im = P[0] * p.y + 2.0f * P[1] * p.x * p.y;
  float r = w / (re * re + im * im);
  return f2((p.x * re + p.y * im) * r, (p.y * re - p.x * im) * r);
}
VAR(rectangles) {  // P = x, y
  float rx = P[0] == 0.0f ? 1.0f : P[0], ry = P[1] == 0.0f ? 1.0f : P[1];
  float ox = P[0] == 0.0f ? w * p.x : w * ((2.0f * floorf(p.x / rx) + 1.0f) * rx - p.x);
  float oy = P[1] == 0.0f ? w * p.y : w * ((2.0f * floorf(p.y / ry) + 1.0f) * ry - p.y);
  return f2(ox, oy);
}
VAR(blob) {  // P = low, high, waves
  float r0 = len2(p), re = r0 + P_EPS;
  float r = r0 * (P[0] + (P[1] - P[0]) * (0.5f + 0.5f * ssin(P[2] * atan2f(p.x, p.y))));
  float k = w * r;
  return f2(k * (p.x / re), k * (p.y / re));
}
VAR(ngon) {  // P = sides, power, circle, corners
  float rf = wpow(sq2(p), P[1] * 0.5f);
  float th = atan2f(p.y, p.x), b = P_TAU / P[0];
  float ph = th - b * floorf(th / b);
  if (ph > b * 0.5f) ph -= b;
  float amp = (P[3] * (1.0f / (scos(ph) + P_EPS) - 1.0f) + P[2]) / (rf + P_EPS);
  return p * (w * amp);
}
VAR(wedge) {  // P = angle, hole, count, swirl
  const float inv_pi = 1.0f / P_PI;
  float r0 = len2(p);
  float a = atan2f(p.y, p.x) + P[3] * r0;
  float k = floorf((P[2] * a + P_PI) * inv_pi * 0.5f);
  a = a * (1.0f - P[0] * P[2] * inv_pi * 0.5f) + k * P[0];
  return polar2(w * (r0 + P[1]), a);
}
VAR(cpow) {  // P = r, i, power
  float a = atan2f(p.y, p.x), lnr = 0.5f * logf(sq2(p));
  float va = P_TAU / P[2], vc = P[0] / P[2], vd = P[1] / P[2];
  float n = floorf(RAND01() * fabsf(P[2]));
  return polar2(w * expf(vc * lnr - vd * a), vc * a + vd * lnr + va * n);
}
VAR(curve) {  // P = xamp, yamp, xlength, ylength
  float lx = fmaxf(P[2] * P[2], 1e-20f), ly = fmaxf(P[3] * P[3], 1e-20f);
  return f2(w * (p.x + P[0] * expf((-p.y * p.y) / lx)), w * (p.y + P[1] * expf((-p.x * p.x) / ly)));
}
VAR(noise) {
  float ang = RAND01() * P_TAU;
  float r = w * RAND01(), s, co;
  ssincos(ang, &s, &co);
  return f2(p.x * r * co, p.y * r * s);
}
VAR(blur) {
  float ang = RAND01() * P_TAU;
  return polar2(w * RAND01(), ang);
}
VAR(gaussian_blur) {
  float ang = RAND01() * P_TAU;
  float g0 = RAND01(), g1 = RAND01(), g2 = RAND01(), g3 = RAND01();
  return polar2(w * (g0 + g1 + g2 + g3 - 2.0f), ang);
}
VAR(arch) {
  float s, co;
  ssincos(RAND01() * w * P_PI, &s, &co);
  return f2(w * s, w * (s * s) / co);
}
VAR(radial_blur) {  // P = angle
  float ang = P[0] * (P_PI * 0.5f), spin = ssin(ang), zoom = scos(ang);
  float g0 = RAND01(), g1 = RAND01(), g2 = RAND01(), g3 = RAND01();
  float g = w * (g0 + g1 + g2 + g3 - 2.0f);
  float ra = len2(p), s, co;
  ssincos(atan2f(p.y, p.x) + spin * g, &s, &co);
  float rz = zoom * g - 1.0f;
  return f2(ra * co + rz * p.x, ra * s + rz * p.y);
}
VAR(juliascope) {  // P = power, dist
  float ph = atan2f(p.y, p.x);
  i32 t = f2i(floorf(RAND01() * fabsf(P[0])));
  float tr = (t & 1) == 0 ? (P_TAU * (float)t + ph) / P[0] : (P_TAU * (float)t - ph) / P[0];
  return polar2(w * wpow(sq2(p), P[1] / P[0] / 2.0f), tr);
}
VAR(square) {
  float u = RAND01(), v = RAND01();
  return f2(w * (u - 0.5f), w * (v - 0.5f));
}
VAR(rays) {
  float ang = w * RAND01() * P_PI;
  float r = w / (sq2(p) + P_EPS);
  float t = w * stan(ang) * r;
  return f2(t * scos(p.x), t * ssin(p.y));
}
VAR(blade) {
  float s, co;
  ssincos(RAND01() * w * len2(p), &s, &co);
  return f2(w * p.x * (co + s), w * p.x * (co - s));
}
VAR(twintrian) {
  float s, co;
  ssincos(RAND01() * w * len2(p), &s, &co);
  float d = logf(s * s) / P_LN10 + co;
  if (d != d || d > 1e10f || d < -1e10f) d = -30.0f;
  return f2(w * p.x * d, w * p.x * (d - s * P_PI));
}
VAR(exp) { return polar2(w * expf(p.x), p.y); }
VAR(log) { return f2(w * (0.5f * logf(sq2(p))), w * atan2f(p.y, p.x)); }
VAR(sin) { return f2(w * (ssin(p.x) * coshf(p.y)), w * (scos(p.x) * sinhf(p.y))); }
VAR(cos) { return f2(w * (scos(p.x) * coshf(p.y)), w * (-ssin(p.x) * sinhf(p.y))); }
VAR(tan) {
  float k = w * (1.0f / (scos(2.0f * p.x) + coshf(2.0f * p.y)));
  return f2(k * ssin(2.0f * p.x), k * sinhf(2.0f * p.y));
}
VAR(sec) {
  float k = w * (2.0f / (scos(2.0f * p.x) + coshf(2.0f * p.y)));
  return f2(k * (scos(p.x) * coshf(p.y)), k * (ssin(p.x) * sinhf(p.y)));
}
VAR(csc) {
  float k = w * (2.0f / (coshf(2.0f * p.y) - scos(2.0f * p.x)));
  return f2(k * (ssin(p.x) * coshf(p.y)), k * (-scos(p.x) * sinhf(p.y)));
}
VAR(cot) {
  float k = w * (1.0f / (coshf(2.0f * p.y) - scos(2.0f * p.x)));
  return f2(k * ssin(2.0f * p.x), k * -sinhf(2.0f * p.y));
}
VAR(sinh) { return f2(w * (sinhf(p.x) * scos(p.y)), w * (coshf(p.x) * ssin(p.y))); }
VAR(cosh) { return f2(w * (coshf(p.x) * scos(p.y)), w * (sinhf(p.x) * ssin(p.y))); }
VAR(tanh) {
  float k = w * (1.0f / (scos(2.0f * p.y) + coshf(2.0f * p.x)));
  return f2(k * sinhf(2.0f * p.x), k * ssin(2.0f * p.y));
}
VAR(sech) {
  float k = w * (2.0f / (scos(2.0f * p.y) + coshf(2.0f * p.x)));
  return f2(k * (scos(p.y) * coshf(p.x)), k * (-ssin(p.y) * sinhf(p.x)));
}
VAR(csch) {
  float k = w * (2.0f / (coshf(2.0f * p.x) - scos(2.0f * p.y)));
  return f2(k * (sinhf(p.x) * scos(p.y)), k * (-coshf(p.x) * ssin(p.y)));
}
VAR(coth) {
  float k = w * (1.0f / (coshf(2.0f * p.x) - scos(2.0f * p.y)));
  return f2(k * sinhf(2.0f * p.x), k * ssin(2.0f * p.y));
}
VAR(butterfly) {
  float y2 = p.y * 2.0f;
  float r = (w * 1.3029400317411197908970256609023f) *
            sqrtf(fabsf(p.y * p.x) / (P_EPS + p.x * p.x + y2 * y2));
  return f2(r * p.x, r * y2);
}
VAR(edisc) {
  float t = sq2(p) + 1.0f, t2 = 2.0f * p.x;
  float xmax = (sqrtf(t + t2) + sqrtf(t - t2)) * 0.5f;
  float a1 = logf(xmax + sqrtf(fmaxf(xmax - 1.0f, 0.0f)));
  float a2 = -acosf(wclamp(p.x / xmax, -1.0f, 1.0f));
  float wn = w / 11.57034632f, s, co;
  ssincos(a1, &s, &co);
  if (p.y > 0.0f) s = -s;
  return f2(wn * coshf(a2) * co, wn * sinhf(a2) * s);
}
VAR(elliptic) {
  float t = sq2(p) + 1.0f, x2 = 2.0f * p.x;
  float xmax = 0.5f * (sqrtf(t + x2) + sqrtf(t - x2));
  float a = p.x / xmax;
  float b = sqrtf(fmaxf(1.0f - a * a, 0.0f)), ssx = sqrtf(fmaxf(xmax - 1.0f, 0.0f));
  float wn = w / (P_PI * 0.5f), yl = wn * logf(xmax + ssx);
  return f2(wn * atan2f(a, b), p.y > 0.0f ? yl : -yl);
}
VAR(foci) {
  float ex = expf(p.x) * 0.5f, enx = 0.25f / ex;
  float s, co;
  ssincos(p.y, &s, &co);
  float t = w / (ex + enx - co);
  return f2(t * (ex - enx), t * s);
}
VAR(loonie) {
  float r2 = sq2(p), w2 = w * w;
  if (r2 < w2) return p * (w * sqrtf(w2 / r2 - 1.0f));
  return p * w;
}
VAR(polar2) {
  float k = w / P_PI;
  return f2(k * atan2f(p.x, p.y), (k * 0.5f) * logf(sq2(p) + P_EPS));
}
VAR(scry) {
  float s = sq2(p);
  return p * (1.0f / (sqrtf(s) * (s + 1.0f / (w + P_EPS))));
}
VAR(bent2) {  // P = x, y
  return f2(w * (p.x < 0.0f ? p.x * P[0] : p.x), w * (p.y < 0.0f ? p.y * P[1] : p.y));
}
VAR(cell) {  // P = size
  const float sz = P[0], inv = 1.0f / sz;
  i32 x = f2i(floorf(p.x * inv)), y = f2i(floorf(p.y * inv));
  float dx = p.x - (float)x * sz, dy = p.y - (float)y * sz;
  y = y >= 0 ? y * 2 : -(2 * y + 1);
  x = x >= 0 ? x * 2 : -(2 * x + 1);
  return f2(w * (dx + (float)x * sz), -w * (dy + (float)y * sz));
}
VAR(escher) {  // P = beta
  float a = atan2f(p.y, p.x), lnr = 0.5f * logf(sq2(p));
  float sb, cb;
  ssincos(P[0], &sb, &cb);
  float vc = 0.5f * (1.0f + cb), vd = 0.5f * sb;
  return polar2(w * expf(vc * lnr - vd * a), vc * a + vd * lnr);
}
VAR(modulus) {  // P = x, y
  const float mx = P[0], my = P[1], xr = 2.0f * mx, yr = 2.0f * my;
  float ox = p.x > mx ? w * (-mx + wmod(p.x + mx, xr))
           : (p.x < -mx ? w * (mx - wmod(mx - p.x, xr)) : w * p.x);
  float oy = p.y > my ? w * (-my + wmod(p.y + my, yr))
           : (p.y < -my ? w * (my - wmod(my - p.y, yr)) : w * p.y);
  return f2(ox, oy);
}
VAR(split) {  // P = xsize, ysize
  float oy = scos(p.x * P[0] * P_PI) >= 0.0f ? w * p.y : -w * p.y;
  float ox = scos(p.y * P[1] * P_PI) >= 0.0f ? w * p.x : -w * p.x;
  return f2(ox, oy);
}
VAR(splits) {  // P = x, y
  return f2(p.x >= 0.0f ? w * (p.x + P[0]) : w * (p.x - P[0]),
            p.y >= 0.0f ? w * (p.y + P[1]) : w * (p.y - P[1]));
}
VAR(stripes) {  // P = space, warp
  float rx = floorf(p.x + 0.5f), ox = p.x - rx;
  return f2(w * (ox * (1.0f - P[0]) + rx), w * (p.y + ox * ox * P[1]));
}
VAR(whorl) {  // P = inside, outside
  float r = len2(p), a0 = atan2f(p.y, p.x);
  float a = r < w ? a0 + P[0] / (w - r) : a0 + P[1] / (w - r);
  return polar2(w * r, a);
}
VAR(flux) {  // P = spread
  float xp = p.x + w, xm = p.x - w, ty = p.y * p.y;
  float r = w * (2.0f + P[0]) * sqrtf(sqrtf(ty + xp * xp) / sqrtf(ty + xm * xm));
  return polar2(r, (atan2f(p.y, xm) - atan2f(p.y, xp)) * 0.5f);
}
VAR(popcorn2) {  // P = x, y, c
  return f2(w * (p.x + P[0] * ssin(stan(p.y * P[2]))), w * (p.y + P[1] * ssin(stan(p.x * P[2]))));
}
VAR(lazysusan) {  // P = x, y, spin, twist, space
  float x = p.x - P[0], y = p.y + P[1], r0 = len2(f2(x, y));
  if (r0 < w) {
    float2 q = polar2(w * r0, atan2f(y, x) + P[2] + P[3] * (w - r0));
    return f2(q.x + P[0], q.y - P[1]);
  }
  float r = w * (1.0f + P[4] / r0);
  return f2(r * x + P[0], r * y - P[1]);
}
VAR(waves2) {  // P = scalex, freqx, scaley, freqy
  return f2(w * (p.x + P[0] * ssin(p.y * P[1])), w * (p.y + P[2] * ssin(p.x * P[3])));
}
VAR(oscilloscope) {  // P = frequency, amplitude, damping, separation
  float tpf = P_TAU * P[0];
  float t = P[2] == 0.0f ? P[1] * scos(tpf * p.x) + P[3]
                         : P[1] * expf(-fabsf(p.x) * P[2]) * scos(tpf * p.x) + P[3];
  if (fabsf(p.y) <= t) return f2(w * p.x, -w * p.y);
  return p * w;
}
VAR(separation) {  // P = x, xinside, y, yinside
  float sx2 = P[0] * P[0], sy2 = P[2] * P[2];
  float hx = sqrtf(p.x * p.x + sx2), hy = sqrtf(p.y * p.y + sy2);
  return f2(p.x > 0.0f ? w * (hx - p.x * P[1]) : -w * (hx + p.x * P[1]),
            p.y > 0.0f ? w * (hy - p.y * P[3]) : -w * (hy + p.y * P[3]));
}
VAR(auger) {  // P = freq, weight, scale, sym
  float s = ssin(P[0] * p.x), t = ssin(P[0] * p.y);
  float dy = p.y + P[1] * (P[2] * s * 0.5f + fabsf(p.y) * s);
  float dx = p.x + P[1] * (P[2] * t * 0.5f + fabsf(p.x) * t);
  return f2(w * (p.x + P[3] * (dx - p.x)), w * dy);
}
VAR(wedge_sph) {  // P = angle, hole, count, swirl
  const float inv_pi = 1.0f / P_PI;
  float ri = 1.0f / (len2(p) + P_EPS);
  float a = atan2f(p.y, p.x) + P[3] * ri;
  float k = floorf((P[2] * a + P_PI) * inv_pi * 0.5f);
  a = a * (1.0f - P[0] * P[2] * inv_pi * 0.5f) + k * P[0];
  return polar2(w * (ri + P[1]), a);
}
VAR(super_shape) {  // P = rnd, m, n1, n2, n3, holes
  float r0 = len2(p);
  float th = P[1] * 0.25f * atan2f(p.y, p.x) + P_PI * 0.25f, s, co;
  ssincos(th, &s, &co);
  float t1 = wpow(fabsf(co), P[3]), t2 = wpow(fabsf(s), P[4]);
  float r = w * ((P[0] * RAND01() + (1.0f - P[0]) * r0) - P[5]) * wpow(t1 + t2, -1.0f / P[2]) / r0;
  return p * r;
}
VAR(flower) {  // P = petals, holes
  float th = atan2f(p.y, p.x), r0 = len2(p);
  return p * (w * (RAND01() - P[1]) * scos(P[0] * th) / r0);
}
VAR(conic) {  // P = eccentricity, holes
  float r0 = len2(p), ct = p.x / r0;
  return p * (w * (RAND01() - P[1]) * P[0] / (1.0f + P[0] * ct) / r0);
}
VAR(parabola) {  // P = height, width
  float s, co;
  ssincos(len2(p), &s, &co);
  float u = RAND01(), v = RAND01();
  return f2(P[0] * w * s * s * u, P[1] * w * co * v);
}
VAR(pie) {  // P = slices, rotation, thickness
  float u = RAND01(), v = RAND01(), t = RAND01();
  float sl = truncf(u * P[0] + 0.5f);
  return polar2(w * t, P[1] + P_TAU * (sl + v * P[2]) / P[0]);
}
VAR(boarders) {
  float u = RAND01();
  float rx = floorf(p.x + 0.5f), ry = floorf(p.y + 0.5f);
  float ox = p.x - rx, oy = p.y - ry;
  float bx = ox * 0.5f + rx, by = oy * 0.5f + ry;
  if (u >= 0.75f) return f2(w * bx, w * by);
  if (fabsf(ox) >= fabsf(oy)) {
    if (ox >= 0.0f) return f2(w * (bx + 0.25f), w * (by + 0.25f * oy / ox));
    return f2(w * (bx - 0.25f), w * (by - 0.25f * oy / ox));
  }
  if (oy >= 0.0f) return f2(w * (bx + ox / oy * 0.25f), w * (by + 0.25f));
  return f2(w * (bx - ox / oy * 0.25f), w * (by - 0.25f));
}
VAR(wedge_julia) {  // P = angle, count, power, dist
  float r = w * wpow(sq2(p), P[3] / P[2] * 0.5f);
  float cf = 1.0f - P[0] * P[1] / P_TAU;
  float n = floorf(RAND01() * fabsf(P[2]));
  float a = (atan2f(p.y, p.x) + P_TAU * n) / P[2];
  float k = floorf((P[1] * a + P_PI) / P_PI * 0.5f);
  return polar2(r, a * cf + k * P[0]);
}
VAR(mobius) {  // P = re_a, im_a, re_b, im_b, re_c, im_c, re_d, im_d
  float ur = P[0] * p.x - P[1] * p.y + P[2], ui = P[0] * p.y + P[1] * p.x + P[3];
  float vr = P[4] * p.x - P[5] * p.y + P[6], vi = P[4] * p.y + P[5] * p.x + P[7];
  float k = w / (vr * vr + vi * vi);
  return f2(k * (ur * vr + ui * vi), k * (ui * vr - ur * vi));
}
