// pyr3-b200 variation library, part 2: direct-colour family (99..102) and
// the first plugin / JWildfire batch (103..127), restated from the
// reference's src/shaders/chaos.wgsl lines 1662-2840 and noise_perlin.wgsl.
#pragma once

// ------------------------------------------------------------ Perlin noise
// 2-D improved Perlin noise with an 8-direction gradient set and fBm
// (noise_perlin.wgsl:48-96); the permutation table c_perlin_perm is emitted
// by the build from the reference's table.
VDEV float perlin_fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }
VDEV float perlin_grad(u32 h, float x, float y) {
  h &= 7u;
  float u = h < 4u ? x : y, v = h < 4u ? y : x;
  return ((h & 1u) ? -u : u) + ((h & 2u) ? -2.0f * v : 2.0f * v);
}
VDEV u32 perm(u32 i) { return (u32)c_perlin_perm[i & 255u]; }
VDEV float perlin2(float px, float py) {
  float fx = floorf(px), fy = floorf(py);
  u32 X = (u32)(f2i(fx) & 255), Y = (u32)(f2i(fy) & 255);
  float xf = px - fx, yf = py - fy;
  float u = perlin_fade(xf), v = perlin_fade(yf);
  u32 A = (perm(X) + Y) & 255u, B = (perm(X + 1u) + Y) & 255u;
  float g00 = perlin_grad(perm(A), xf, yf);
  float g10 = perlin_grad(perm(B), xf - 1.0f, yf);
  float g01 = perlin_grad(perm(A + 1u), xf, yf - 1.0f);
  float g11 = perlin_grad(perm(B + 1u), xf - 1.0f, yf - 1.0f);
  return wmix(wmix(g00, g10, u), wmix(g01, g11, u), v);
}
VDEV float perlin_fbm(float2 p, float octaves, float scale) {
  float total = 0.0f, amp = 1.0f, freq = scale, maxv = 0.0f;
  u32 n = f2u(wclamp(octaves, 1.0f, 8.0f));
  for (u32 i = 0; i < n; ++i) {
    total += perlin2(p.x * freq, p.y * freq) * amp;
    maxv += amp;
    amp *= 0.5f;
    freq *= 2.0f;
  }
  return total / maxv;
}

// ------------------------------------------------------- direct colour
DCV(dc_linear) {
  return make_float3(wclamp(0.5f + 0.5f * p.x, 0.0f, 1.0f), wclamp(0.5f + 0.5f * p.y, 0.0f, 1.0f),
                     wclamp(0.5f - 0.25f * (p.x + p.y), 0.0f, 1.0f));
}
DCV(dc_perlin) {  // P = scale, octaves, color_seed
  float n = perlin_fbm(p, P[1], fmaxf(P[0], 1e-6f));
  return hsl_rgb(wfract(0.5f + 0.5f * n + P[2]), 1.0f, 0.55f);
}
DCV(dc_gridout) {  // P = cells
  float n = fmaxf(P[0], 1.0f);
  i32 cx = f2i(floorf(p.x * n)), cy = f2i(floorf(p.y * n));
  u32 m = (u32)((cx * 73856093) ^ (cy * 19349663)) + 0x9e3779b9u;
  return make_float3(hash01(m), hash01(m ^ 0xdeadbeefu), hash01(m ^ 0x13579bdfu));
}
DCV(dc_cylinder) {
  float hue = wfract(0.5f + 0.5f * ssin(p.x));
  float lit = wclamp(0.5f + 0.25f * stanh(p.y * 0.5f), 0.2f, 0.85f);
  return hsl_rgb(hue, 0.9f, lit);
}
VAR(dc_cylinder) { return f2(w * ssin(p.x), w * p.y); }

// ------------------------------------------------------------- 103..127
VAR(cpow2) {  // P = r, a, divisor, range
  float div = P[2] == 0.0f ? 1.0f : P[2];
  float rmax = fmaxf(P[3], 1.0f);
  float step = P_TAU / div;
  float cc = P[0] * scos(P_PI * 0.5f * P[1]) / div;
  float dd = P[0] * ssin(P_PI * 0.5f * P[1]) / div;
  float u0 = RAND01(), u1 = RAND01(), u2 = RAND01();
  float a = atan2f(p.y, p.x);
  a += P_TAU * (floorf(u0 * rmax) + (a < 0.0f ? 1.0f : 0.0f));
  if (scos(a * (0.5f / rmax)) < (u1 * 2.0f - 1.0f)) a -= P_TAU * rmax;
  float lnr2 = logf(sq2(p));
  float r = w * expf(cc * 0.5f * lnr2 - dd * a);
  return polar2(r, cc * a + (dd * 0.5f) * lnr2 + step * floorf(div * u2));
}
VAR(cpow3) {  // P = r, d, divisor, spread
  float div = P[2] == 0.0f ? 1.0f : P[2];
  float step = P_TAU / div;
  float dab = fmaxf(fabsf(P[1]), 1e-30f);
  float sl = P[1] < 0.0f ? -logf(dab) : logf(dab);
  float pa = atan2f(sl * P[0], P_TAU);
  float cpa = scos(pa), spa = ssin(pa);
  float tc = cpa * P[0] * cpa / div, td = cpa * P[0] * spa / div;
  float coeff = td == 0.0f ? 0.0f : -0.095f * P[3] / td;
  float u0 = RAND01(), u1 = RAND01(), u2 = RAND01(), u3 = RAND01();
  float a = atan2f(p.y, p.x);
  if (a < 0.0f) a += P_TAU;
  if (scos(a * 0.5f) < (u0 * 2.0f - 1.0f)) a -= P_TAU;
  a += (u1 < 0.5f ? P_TAU : -P_TAU) * wround(logf(fmaxf(u2, 1e-30f)) * coeff);
  float lnr2 = logf(sq2(p));
  float r = w * expf(tc * 0.5f * lnr2 - td * a);
  return polar2(r, tc * a + td * 0.5f * lnr2 + step * floorf(div * u3));
}
VAR(loonie2) {  // P = sides, star, circle
  const i32 kMax = 16;
  i32 sides = min(max(f2i(P[0]), 1), kMax);
  float sa, ca;
  ssincos(P_TAU / (float)sides, &sa, &ca);
  float sins = ssin(-P[1] * P_PI * 0.5f), coss = scos(P[1] * P_PI * 0.5f);
  float sinc = ssin(P[2] * P_PI * 0.5f), cosc = scos(P[2] * P_PI * 0.5f);
  float sqv = w * w;
  float xr = p.x, yr = p.y;
  float r2 = xr * coss + fabsf(yr) * sins;
  float cr = sqrtf(xr * xr + yr * yr);
  for (i32 i = 0; i < kMax && i < sides - 1; ++i) {
    float sw = xr * ca - yr * sa;
    yr = xr * sa + yr * ca;
    xr = sw;
    r2 = fmaxf(r2, xr * coss + fabsf(yr) * sins);
  }
  r2 = r2 * cosc + cr * sinc;
  r2 = sides > 2 ? r2 * r2 : fabsf(r2) * r2;
  if (r2 > 0.0f && r2 < sqv) return p * (w * sqrtf(fabsf(sqv / r2 - 1.0f)));
  if (r2 < 0.0f) return p * (w / sqrtf(fabsf(sqv / r2) - 1.0f));
  return p * w;
}
VAR(epispiral) {  // P = n, thickness, holes
  float th = atan2f(p.y, p.x);
  float d = scos(P[0] * th);
  float u = RAND01();
  float rc = 1.0f / d;
  float t = fabsf(P[1]) > 1e-30f ? -P[2] + (u * P[1]) * rc : -P[2] + rc;
  float s, co;
  ssincos(th, &s, &co);
  return f2(w * t * co, w * t * s);
}

// Worley cell feature point (chaos.wgsl:1933-1946).
VDEV float2 worley_hash(i32 cx, i32 cy) {
  u32 s = (u32)cx * 2654435769u;
  s ^= (u32)cy * 2246822519u;
  s ^= s >> 16; s *= 0x85ebca6bu;
  s ^= s >> 13; s *= 0xc2b2ae35u;
  s ^= s >> 16;
  return f2((float)(s & 0xffffu) * (1.0f / 65535.0f), (float)((s >> 16) & 0xffffu) * (1.0f / 65535.0f));
}
VAR(bwraps) {  // P = cellsize, space, gain, inner_twist, outer_twist
  const float cs = P[0];
  if (fabsf(cs) < 1e-30f) return p * w;
  float rad = 0.5f * (cs / (1.0f + P[1] * P[1]));
  float g2 = P[2] * P[2] / cs + 1e-6f;
  float mb = g2 * rad;
  mb = mb > 2.0f ? 1.0f : mb * (1.0f / ((mb * mb) / 4.0f + 1.0f));
  float rr2 = rad * rad, rfac = rad / fmaxf(mb, 1e-30f);
  float cx = (floorf(p.x / cs) + 0.5f) * cs, cy = (floorf(p.y / cs) + 0.5f) * cs;
  float lx = p.x - cx, ly = p.y - cy;
  if (lx * lx + ly * ly > rr2) return p * w;
  lx *= g2;
  ly *= g2;
  float rd = rfac / ((lx * lx + ly * ly) / 4.0f + 1.0f);
  lx *= rd;
  ly *= rd;
  float rf = (lx * lx + ly * ly) / fmaxf(rr2, 1e-30f);
  float st, ct;
  ssincos(P[3] * (1.0f - rf) + P[4] * rf, &st, &ct);
  return f2(w * (cx + ct * lx + st * ly), w * (cy - st * lx + ct * ly));
}
VDEV float2 crackle_centre(i32 cx, i32 cy, float s, float d) {
  float fx = (float)cx, fy = (float)cy;
  float ex = perlin2(fx * 2.5f, fy * 2.5f);
  float ey = perlin2(fy * 2.5f + 30.2f, fx * 2.5f - 12.1f);
  return f2((fx + d * ex) * s, (fy + d * ey) * s);
}
VDEV float crackle_ratio(float2 a, float2 q, float2 u) {
  float2 d = a - q;
  float den = d.x * d.x + d.y * d.y;
  if (den < 1e-30f) return 1.0f;
  return 2.0f * ((u.x - q.x) * d.x + (u.y - q.y) * d.y) / den;
}
VAR(crackle) {  // P = cellsize, power, distort, scale
  if (fabsf(P[0]) < 1e-30f) return p * w;
  float s = P[0] * 0.5f;
  float u1 = RAND01(), u2 = RAND01(), u3 = RAND01(), u4 = RAND01();
  float bl = (u1 + u2) * 0.5f + (u3 - 0.5f) * 0.25f;
  float th = 2.0f * P_PI * u4;
  float2 u = f2(bl * sinf(th), bl * cosf(th));
  i32 x0 = f2i(floorf(u.x / s)), y0 = f2i(floorf(u.y / s));
  float best = 1e30f;
  int q = 0;
  for (int i = 0; i < 9; ++i) {
    float2 c0 = crackle_centre(x0 + i / 3 - 1, y0 + i % 3 - 1, s, P[2]);
    float d2 = (c0.x - u.x) * (c0.x - u.x) + (c0.y - u.y) * (c0.y - u.y);
    if (d2 < best) { best = d2; q = i; }
  }
  i32 xc = x0 + q / 3 - 1, yc = y0 + q % 3 - 1;
  float2 ctr = crackle_centre(xc, yc, s, P[2]);
  float L = -1e30f;
  for (int i = 0; i < 9; ++i) {
    if (i == 4) continue;
    L = fmaxf(L, crackle_ratio(crackle_centre(xc + i / 3 - 1, yc + i % 3 - 1, s, P[2]), ctr, u));
  }
  float ls = L + 1e-30f;
  float R = wpow(fabsf(ls), P[1]) * P[3] / ls;
  return f2(w * (ctr.x + (u.x - ctr.x) * R), w * (ctr.y + (u.y - ctr.y) * R));
}
VAR(juliaq) {  // P = power, divisor
  float pw = fabsf(P[0]) < 1e-30f ? 1.0f : P[0];
  float ap = fmaxf(1.0f, fabsf(pw));
  float ip = P[1] / pw;
  float n = floorf(RAND01() * ap);
  float a = atan2f(p.y, p.x) * ip + n * (P_TAU / pw);
  return polar2(w * wpow(p.x * p.x + p.y * p.y, 0.5f * ip), a);
}
VAR(glynnia) {
  float v2 = w * 0.7071067811865476f;
  float r = sqrtf(p.x * p.x + p.y * p.y);
  float coin = RAND01();
  const float sgn = r >= 1.0f ? 1.0f : -1.0f;
  if (coin > 0.5f) {
    float in = r + p.x;
    if (in <= 0.0f) return f2(0.0f, 0.0f);
    float d = sqrtf(in);
    if (d == 0.0f) return f2(0.0f, 0.0f);
    return f2(sgn * v2 * d, -(v2 / d) * p.y);
  }
  float d = r + p.x;
  float rad = r * (p.y * p.y + d * d);
  if (rad <= 0.0f) return f2(0.0f, 0.0f);
  float dx = sqrtf(rad);
  if (dx == 0.0f) return f2(0.0f, 0.0f);
  float rr = w / dx;
  return f2(sgn * rr * d, rr * p.y);
}
VAR(loonie3) {
  float sqv = w * w, r2 = 2.0f * sqv;
  if (p.x > 1e-30f) {
    float q = (p.x * p.x + p.y * p.y) / p.x;
    r2 = q * q;
  }
  if (r2 < sqv) return p * (w * sqrtf(sqv / r2 - 1.0f));
  return p * w;
}
VAR(falloff) {  // P = scatter, mindist, mul_x, mul_y, x0, y0
  float rmax = 0.04f * P[0];
  float dx = p.x - P[4], dy = p.y - P[5];
  float d = fmaxf((fmaxf(sqrtf(dx * dx + dy * dy), 0.0f) - P[1]) * rmax, 0.0f);
  float u0 = RAND01(), u1 = RAND01();
  return f2(w * (p.x + P[2] * u0 * d), w * (p.y + P[3] * u1 * d));
}
VAR(falloff2) {  // P = scatter, type, mul_x, mul_y, x0, y0, mindist
  float rmax = 0.04f * P[0];
  float dx = p.x - P[4], dy = p.y - P[5];
  float d = fmaxf((fmaxf(sqrtf(dx * dx + dy * dy), 0.0f) - P[6]) * rmax, 0.0f);
  float u0 = RAND01(), u1 = RAND01(), u2 = RAND01();
  i32 t = f2i(wclamp(P[1], 0.0f, 2.0f));
  if (t == 1) {
    float ra = sqrtf(p.x * p.x + p.y * p.y);
    float ph = atan2f(p.y, p.x) + P[3] * d * u1;
    float rr = ra + P[2] * u0 * d;
    float s, co;
    ssincos(ph, &s, &co);
    return f2(w * rr * co, w * rr * s);
  }
  if (t == 2) {
    float sc = scos(d * u1 * P_TAU), ph = d * u2 * P_PI, rd = d * u0;
    return f2(w * (p.x + P[2] * rd * sc * scos(ph)), w * (p.y + P[3] * rd * sc * ssin(ph)));
  }
  return f2(w * (p.x + P[2] * u0 * d), w * (p.y + P[3] * u1 * d));
}
VAR(falloff3) {  // P = scatter, mul_x, mul_y, x0, y0, mindist, invert
  float rmax = 0.04f * P[0];
  float dx = p.x - P[3], dy = p.y - P[4];
  float rad = sqrtf(dx * dx + dy * dy);
  float base = P[6] > 0.5f ? fmaxf(1.0f - rad, 0.0f) : fmaxf(rad, 0.0f);
  float dist = fmaxf((base - P[5]) * rmax, 0.0f);
  float u0 = RAND01() - 0.5f, u1 = RAND01() - 0.5f, u2 = RAND01() - 0.5f;
  float sc = scos(dist * u1 * P_TAU), ph = dist * u2 * P_PI, rd = dist * u0;
  return f2(w * (p.x + P[1] * rd * sc * scos(ph)), w * (p.y + P[2] * rd * sc * ssin(ph)));
}
VAR(collideoscope) {  // P = a, num
  float nf = (float)max(1, f2i(P[1]));
  float kn_pi = nf / P_PI, pi_kn = P_PI / nf, ka_kn = (P_PI * P[0]) / nf;
  float a = atan2f(p.y, p.x);
  float r = w * sqrtf(p.x * p.x + p.y * p.y);
  if (a >= 0.0f) {
    i32 alt = f2i(a * kn_pi);
    a = (float)alt * pi_kn + wmod(((alt % 2) == 0 ? ka_kn : -ka_kn) + a, pi_kn);
  } else {
    i32 alt = f2i(-a * kn_pi);
    a = -((float)alt * pi_kn + wmod(((alt % 2) != 0 ? -ka_kn : ka_kn) - a, pi_kn));
  }
  return polar2(r, a);
}
// Square-to-circle perimeter mapping shared by circlize / circlize2.
VDEV bool circ_perimeter(float2 p, float* per, float* side) {
  float ax = fabsf(p.x), ay = fabsf(p.y);
  if (ax >= ay) {
    *per = p.x >= ay ? ax + p.y : 5.0f * ax - p.y;
    *side = ax;
  } else {
    *per = p.y >= ax ? 3.0f * ay - p.x : 7.0f * ay + p.x;
    *side = ay;
  }
  return *side != 0.0f;
}
VAR(circlize) {  // P = hole
  float per, side;
  if (!circ_perimeter(p, &per, &side)) return f2(0.0f, 0.0f);
  float r = (w / (P_PI * 0.25f)) * side + P[0];
  return polar2(r, (P_PI * 0.25f) * per / side - (P_PI * 0.25f));
}
VAR(circlize2) {  // P = hole
  float per, side;
  if (!circ_perimeter(p, &per, &side)) return f2(0.0f, 0.0f);
  return polar2(w * (side + P[0]), (P_PI * 0.25f) * per / side - (P_PI * 0.25f));
}
VAR(eswirl) {  // P = in, out
  float t0 = p.y * p.y + p.x * p.x + 1.0f, t2 = 2.0f * p.x;
  float a1 = t0 + t2, a2 = t0 - t2;
  float xmax = ((a1 > 0.0f ? sqrtf(fmaxf(a1, 0.0f)) : 0.0f) + (a2 > 0.0f ? sqrtf(fmaxf(a2, 0.0f)) : 0.0f)) * 0.5f;
  if (xmax < 1.0f) xmax = 1.0f;
  float mu = logf(xmax + sqrtf(fmaxf(xmax * xmax - 1.0f, 0.0f)));
  float nu = acosf(wclamp(p.x / xmax, -1.0f, 1.0f));
  if (p.y < 0.0f) nu = -nu;
  float nw = nu + mu * P[1] + P[0] / (mu == 0.0f ? 1e-30f : mu);
  return f2(w * coshf(mu) * scos(nw), w * sinhf(mu) * ssin(nw));
}
VAR(petal) {
  float sx, cx;
  ssincos(p.x, &sx, &cx);
  float cy = scos(p.y);
  float a = cx * cy, b = sx * cy;
  return f2(w * cx * (a * a * a), w * cx * (b * b * b));
}
VAR(bcircle) {  // P = scale, borderwidth
  float bw = fabsf(P[1]);
  if (p.x == 0.0f && p.y == 0.0f) return f2(0.0f, 0.0f);
  float x = p.x * P[0], y = p.y * P[0];
  if (sqrtf(x * x + y * y) <= 1.0f) return f2(w * x, w * y);
  if (bw == 0.0f) return f2(0.0f, 0.0f);
  float ang = atan2f(y, x);
  float om = 0.2f * bw * RAND01() + 1.0f;
  float s, co;
  ssincos(ang, &s, &co);
  return f2(w * om * co, w * om * s);
}
VAR(curl2) {  // P = c1, c2, c3
  float x = p.x, y = p.y, x2 = x * x, y2 = y * y;
  float re = P[2] * (x2 * x) - (3.0f * P[2]) * x * y2 + P[1] * x2 - P[1] * y2 + P[0] * x + 1.0f;
  float im = (3.0f * P[2]) * x2 * y - P[2] * (y2 * y) + (2.0f * P[1]) * x * y + P[0] * y;
  float r = w / (re * re + im * im);
  return f2((x * re + y * im) * r, (y * re - x * im) * r);
}
VAR(murl) {  // P = c, power
  i32 pi = f2i(P[1]);
  float pf = (float)pi;
  float cc = pi == 1 ? P[0] : P[0] / (pf - 1.0f);
  float vp = w * (cc + 1.0f);
  float sa, ca;
  ssincos(atan2f(p.y, p.x) * pf, &sa, &ca);
  float r = cc * wpow(p.x * p.x + p.y * p.y, pf / 2.0f);
  float re = r * ca + 1.0f, im = r * sa;
  float r1 = vp / (re * re + im * im + 1e-29f);
  return f2(r1 * (p.x * re + p.y * im), r1 * (p.y * re - p.x * im));
}
VAR(stwins) {  // P = distort
  float x = p.x * w * 0.05f, y = p.y * w * 0.05f;
  float x2 = x * x, y2 = y * y, s2 = x2 + y2;
  float res = (x2 - y2) * ssin(P_TAU * P[0] * (x + y)) / (s2 == 0.0f ? 1.0f : s2);
  return f2(w * p.x + res, w * p.y + res);
}

// Hexagonal Voronoi cell helpers (chaos.wgsl:2725-2760).
VDEV float hex_ratio_step(float2 a, float2 q, float ux, float uy, float prev) {
  float dx = a.x - q.x, dy = a.y - q.y;
  if (dx == 0.0f && dy == 0.0f) return 1.0f > prev ? 1.0f : prev;
  float r = (2.0f * ((ux - q.x) * dx + (uy - q.y) * dy)) / (dx * dx + dy * dy);
  return r > prev ? r : prev;
}
VDEV float2 hex_centre(i32 hx, i32 hy, float s) {
  const float c = 1.7320508075688772935f / 2.0f;
  return f2((1.5f * (float)hx + -1.5f * (float)hy) * s, (c * (float)hx + c * (float)hy) * s);
}
VDEV float hex_vmax(const float2* c, float ux, float uy) {
  float m = -1.0e20f;
  for (int k = 1; k < 7; ++k) m = hex_ratio_step(c[k], c[0], ux, uy, m);
  return m;
}
VAR(hexes) {  // P = cellsize, power, rotate, scale
  const float s = P[0];
  if (s == 0.0f) return f2(0.0f, 0.0f);
  const float r3 = 1.7320508075688772935f;
  float rs, rc;
  ssincos(P[2] * P_TAU, &rs, &rc);
  float ux = p.x, uy = p.y;
  i32 h0 = f2i(floorf(((1.0f / 3.0f) * ux + (r3 / 3.0f) * uy) / s));
  i32 k0 = f2i(floorf(((-1.0f / 3.0f) * ux + (r3 / 3.0f) * uy) / s));
  float best = 1e30f;
  int q = 0;
  for (int di = -1; di < 2; ++di)
    for (int dj = -1; dj < 2; ++dj) {
      float2 c0 = hex_centre(h0 + di, k0 + dj, s);
      float dx = c0.x - ux, dy = c0.y - uy, d2 = dx * dx + dy * dy;
      if (d2 < best) { best = d2; q = (di + 1) * 3 + (dj + 1); }
    }
  i32 hx = h0 + q / 3 - 1, hy = k0 + q % 3 - 1;
  float2 cen[7] = {hex_centre(hx, hy, s),         hex_centre(hx, hy + 1, s),     hex_centre(hx + 1, hy + 1, s),
                 hex_centre(hx + 1, hy, s),     hex_centre(hx, hy - 1, s),     hex_centre(hx - 1, hy - 1, s),
                 hex_centre(hx - 1, hy, s)};
  float L1 = hex_vmax(cen, ux, uy);
  float dxo = ux - cen[0].x, dyo = uy - cen[0].y;
  float trg = wpow(L1 + 1e-30f, P[1]) * P[3];
  float vx = dxo * rc + dyo * rs, vy = -dxo * rs + dyo * rc;
  float L2 = hex_vmax(cen, vx + cen[0].x, vy + cen[0].y);
  float L = fmaxf(L1, L2);
  float R = L < 0.5f ? trg / L1 : (L > 0.8f ? trg / L2 : ((trg / L1) * (0.8f - L) + (trg / L2) * (L - 0.5f)) / 0.3f);
  return f2(w * (vx * R + cen[0].x), w * (vy * R + cen[0].y));
}
VAR(xheart) {  // P = angle, ratio
  float ang = P_PI / 4.0f + (0.5f * (P_PI / 4.0f) * P[0]);
  float sa, ca;
  ssincos(ang, &sa, &ca);
  float rat = 6.0f + 2.0f * P[1];
  float r24 = p.x * p.x + p.y * p.y + 4.0f;
  if (r24 == 0.0f) r24 = 1.0f;
  float bx = 4.0f / r24, by = rat / r24;
  float xr = ca * (bx * p.x) - sa * (by * p.y);
  float yr = sa * (bx * p.x) + ca * (by * p.y);
  return f2(w * xr, w * (xr > 0.0f ? yr : -yr));
}
VAR(xhyperbol) {  // P = m00, m01, m10, m11, m20, m21
  float r = 1.0f / (p.x * p.x + p.y * p.y + P_EPS);
  float x = p.x * r, y = p.y * r;
  float re = P[0] * x + P[1] * y + P[4], im = P[2] * x + P[3] * y + P[5];
  float sa, ca;
  ssincos(atan2f(im, re) + P_TAU, &sa, &ca);
  float rq = re * re + im * im;
  float xo = rq * ca, yo = rq * sa;
  float ri = w / (xo * xo + yo * yo + P_EPS);
  return f2(xo * ri, yo * ri);
}
VAR(xcurl2) {  // P = c1, c2, c3
  float x = p.x, y = p.y, x2 = x * x, y2 = y * y;
  float re = 1.0f + P[0] * x + P[1] * (x2 - y2) + P[2] * (x2 * x - 3.0f * x);
  float im = P[0] * y + P[1] * (2.0f * x * y) + P[2] * (3.0f * x * y - 1.0f);
  float r = w / (re * re + im * im);
  return f2((x * re + y * im) * r, (y * re + x * im) * r);
}
