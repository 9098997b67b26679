// pyr3-b200 variation library, part 5: indices 193..222 plus the
// escape-time family 310..313 and their direct colours, restated from the
// reference's src/shaders/chaos.wgsl lines 4633-5540.
#pragma once

VAR(julia_outside) {  // P = re_div, im_div, mode
  i32 mode = f2i(P[2]);
  bool sq = mode == 0 || mode == 2, rt = mode == 0 || mode == 1;
  float2 z = p, z2 = p;
  if (sq) z = csqrt(z);
  z.x += 1.0f;
  if (sq) z = csqr(z);
  if (sq) z2 = csqrt(z2);
  z2.x -= 1.0f;
  if (sq) z2 = csqr(z2);
  z = cdiv(z, z2);
  if (rt) z = csqrt(z);
  z = cdiv(z, f2(P[0], P[1]));
  if (rt) {
    float s = RAND01() < 0.5f ? 1.0f : -1.0f;
    return f2(w * s * z.x, w * s * z.y);
  }
  return f2(w * z.x, w * z.y);
}
VAR(fourth) {  // P = spin, space, twist, x, y
  float sq = w * w;
  if (p.x > 0.0f && p.y > 0.0f) {
    float th = atan2f(p.y, p.x);
    float r = 1.0f / fmaxf(sqrtf(p.x * p.x + p.y * p.y), 1e-30f);
    return f2(w * r * cosf(th), w * r * sinf(th));
  }
  if (p.x > 0.0f && p.y < 0.0f) {
    float r2 = p.x * p.x + p.y * p.y;
    if (r2 < sq) return p * (w * sqrtf(fmaxf(sq / fmaxf(r2, 1e-30f) - 1.0f, 0.0f)));
    return p * w;
  }
  if (p.x < 0.0f && p.y > 0.0f) {
    float x = p.x - P[3], y = p.y + P[4];
    float r0 = sqrtf(x * x + y * y);
    if (r0 < w) {
      float2 q = polar2(w * r0, atan2f(y, x) + P[0] + P[2] * (w - r0));
      return f2(q.x + P[3], q.y - P[4]);
    }
    float r = w * (1.0f + P[1] / fmaxf(r0, 1e-30f));
    return f2(r * x + P[3], r * y - P[4]);
  }
  return p * w;
}
VAR(pulse) {  // P = freqx, freqy, scalex, scaley
  return f2(w * (p.x + P[2] * ssin(p.x * P[0])), w * (p.y + P[3] * ssin(p.y * P[1])));
}
VDEV float nz_or(float v) { return v == 0.0f ? 1e-30f : v; }
VAR(rays1) {
  float t = p.x * p.x + p.y * p.y;
  float tv = stan(sqrtf(fmaxf(t, 1e-30f)));
  float u = 1.0f / (fabsf(tv) < 1e-30f ? 1e-30f : tv) + w * (2.0f / P_PI) * (2.0f / P_PI);
  return f2(w * u * t / nz_or(p.x), w * u * t / nz_or(p.y));
}
VAR(rays2) {
  float t = p.x * p.x + p.y * p.y, ts = fmaxf(t, 1e-30f);
  float ci = scos((ts + 1e-6f) * stan(1.0f / ts + 1e-6f));
  float u = 1.0f / (fabsf(ci) < 1e-30f ? 1e-30f : ci);
  float k = w / 10.0f;
  return f2(k * u * t / nz_or(p.x), k * u * t / nz_or(p.y));
}
VAR(rays3) {
  float t = p.x * p.x + p.y * p.y, ts = fmaxf(t, 1e-30f);
  float in = ssin(t * t + 1e-6f) * ssin(1.0f / (ts * ts) + 1e-6f);
  float u = 1.0f / fmaxf(sqrtf(fmaxf(scos(in), 1e-30f)), 1e-30f);
  float k = w / 10.0f;
  return f2(k * u * scos(t) * t / nz_or(p.x), k * u * stan(t) * t / nz_or(p.y));
}
VAR(tancos) {
  float d1 = 1e-6f + p.x * p.x + p.y * p.y, d2 = w / d1;
  return f2(d2 * stanh(d1) * 2.0f * p.x, d2 * scos(d1) * 2.0f * p.y);
}
VAR(twoface) {
  float v = w;
  if (p.x > 0.0f) v = v / fmaxf(p.x * p.x + p.y * p.y, 1e-30f);
  return p * v;
}
// Elliptic (mu, nu) coordinates shared by the e_* family (chaos.wgsl:4814-4935).
VDEV float ell_xmax(float x, float r2) {
  float t = r2 + 1.0f, t2 = 2.0f * x;
  float xm = (sqrtf(fmaxf(t + t2, 0.0f)) + sqrtf(fmaxf(t - t2, 0.0f))) * 0.5f;
  return xm < 1.0f ? 1.0f : xm;
}
VAR(e_julia) {  // P = power
  float pw = P[0] == 0.0f ? 1.0f : P[0];
  float r2 = p.y * p.y + p.x * p.x, x = p.x;
  if (!(pw > 0.0f)) {
    r2 = 1.0f / fmaxf(r2, 1e-30f);
    x = p.x * r2;
  }
  float xm = ell_xmax(x, r2);
  float mu0 = acoshf(xm);
  float nu = acosf(wclamp(x / xm, -1.0f, 1.0f));
  if (p.y < 0.0f) nu = -nu;
  float k = floorf(RAND01() * fabsf(pw));
  nu = nu / pw + (2.0f * P_PI / pw) * k;
  float mu = mu0 / pw;
  return f2(w * coshf(mu) * scos(nu), w * sinhf(mu) * ssin(nu));
}
VAR(cannabis_curve_wf) {  // P = filled
  float a = atan2f(p.y, p.x);
  float r = (1.0f + 0.9f * cosf(8.0f * a)) * (1.0f + 0.1f * cosf(24.0f * a)) *
            (0.9f + 0.1f * cosf(200.0f * a)) * (1.0f + sinf(a));
  a += P_PI * 0.5f;
  if (P[0] > 0.0f && P[0] > RAND01()) r *= RAND01();
  return f2(w * sinf(a) * r, w * cosf(a) * r);
}
VAR(e_collide) {  // P = num, a
  float num = fmaxf(1.0f, P[0]);
  float k_pi = num / P_PI, pi_k = P_PI / num, ak = P_PI * P[1] / num;
  float xm = ell_xmax(p.x, p.y * p.y + p.x * p.x);
  float nu = acosf(wclamp(p.x / xm, -1.0f, 1.0f));
  i32 alt = f2i(nu * k_pi);
  float arg = nu + ((alt & 1) == 0 ? ak : -ak);
  nu = (float)alt * pi_k + (arg - floorf(arg / pi_k) * pi_k);
  if (p.y <= 0.0f) nu = -nu;
  return f2(w * xm * cosf(nu), w * sqrtf(fmaxf(xm - 1.0f, 0.0f)) * sqrtf(xm + 1.0f) * sinf(nu));
}
VAR(e_mod) {  // P = radius, distance
  float xm = ell_xmax(p.x, p.y * p.y + p.x * p.x);
  float mu = acoshf(xm);
  float nu = acosf(wclamp(p.x / xm, -1.0f, 1.0f));
  if (p.y < 0.0f) nu = -nu;
  if (mu < P[0] && -mu < P[0]) {
    float rs = fmaxf(P[0], 1e-30f), tr = 2.0f * rs;
    mu = nu > 0.0f ? wmod(mu + rs + P[1] * rs, tr) - rs : wmod(mu - rs - P[1] * rs, tr) + rs;
  }
  return f2(w * coshf(mu) * cosf(nu), w * sinhf(mu) * sinf(nu));
}
VAR(intersection) {  // P = xwidth, xtilesize, xmod1, xmod2, xheight, yheight, ytilesize, ymod1, ymod2, ywidth
  if (w == 0.0f) return f2(0.0f, 0.0f);
  if (RAND01() < 0.5f) {
    float x = RAND01() < 0.5f ? P[0] : -P[0];
    float ox = P[1] * (p.x + wround(x * logf(fmaxf(RAND01(), 1e-30f))));
    float m1 = P[2], r1 = fmaxf(P[3] * P[2], 1e-30f), oy;
    if (p.y > m1) oy = P[4] * (-m1 + wmod(p.y + m1, r1));
    else if (p.y < -m1) oy = P[4] * (m1 - wmod(m1 - p.y, r1));
    else oy = P[4] * p.y;
    return f2(ox, oy);
  }
  float y = RAND01() < 0.5f ? P[5] : -P[5];
  float oy = P[6] * (p.y + wround(y * logf(fmaxf(RAND01(), 1e-30f))));
  float m1 = P[7], r1 = fmaxf(P[8] * P[7], 1e-30f), ox;
  if (p.x > m1) ox = P[9] * (-m1 + wmod(p.x + m1, r1));
  else if (p.x < -m1) ox = P[9] * (m1 - wmod(m1 - p.x, r1));
  else ox = P[9] * p.x;
  return f2(ox, oy);
}
VAR(inv_squircular) {
  if (w == 0.0f) return f2(0.0f, 0.0f);
  float u = p.x, v = p.y, ri = u * u + v * v;
  float r2 = sqrtf(fmaxf(ri * (w * w * ri - 4.0f * u * u * v * v) / w, 0.0f));
  float r = sqrtf(fmaxf(ri - r2, 0.0f)) / 1.41421356237f;
  return f2(r / nz_or(u), r / nz_or(v));
}
VAR(lozi) { return f2(w * (P[2] - P[0] * fabsf(p.x) + p.y), w * P[1] * p.x); }  // P = a, b, c
VAR(hypershift) {  // P = shift, stretch
  float sc = 1.0f - P[0] * P[0];
  float r1 = 1.0f / fmaxf(p.x * p.x + p.y * p.y, 1e-30f);
  float x = r1 * p.x + P[0], y = r1 * p.y;
  float rad = w * sc / fmaxf(x * x + y * y, 1e-30f);
  return f2(rad * x + P[0], rad * y * P[1]);
}
VAR(hex_modulus) {  // P = size
  const float s32 = 0.8660254037844386f, s3 = 1.7320508075688772f;
  float hs = s32 / fmaxf(P[0], 1e-30f), wt = w / s32;
  float X = p.x * hs, Y = p.y * hs;
  float x = 0.5773502691896258f * X - Y / 3.0f, z = 2.0f * Y / 3.0f, y = -x - z;
  float rx = wround(x), ry = wround(y), rz = wround(z);
  float dx = fabsf(rx - x), dy = fabsf(ry - y), dz = fabsf(rz - z);
  if (dx > dy && dx > dz) rx = -ry - rz;
  else if (dy > dz) ry = -rx - rz;
  else rz = -rx - ry;
  return f2((X - (s3 * rx + s32 * rz)) * wt, (Y - 1.5f * rz) * wt);
}
VAR(boarders2) {  // P = c, left, right
  float c0 = fmaxf(fabsf(P[0]), 1e-6f), al = fmaxf(fabsf(P[1]), 1e-6f), ar = fmaxf(fabsf(P[2]), 1e-6f);
  float cl = c0 * al, cr = c0 + c0 * ar;
  float rx = wround(p.x), ry = wround(p.y);
  float ox = p.x - rx, oy = p.y - ry;
  float bx = ox * c0 + rx, by = oy * c0 + ry;
  if (RAND01() >= cr) return f2(w * bx, w * by);
  if (fabsf(ox) >= fabsf(oy)) {
    if (ox >= 0.0f) return f2(w * (bx + cl), w * (by + cl * oy / nz_or(ox)));
    return f2(w * (bx - cl), w * (by - cl * oy / nz_or(ox)));
  }
  if (oy >= 0.0f) return f2(w * (bx + ox / nz_or(oy) * cl), w * (by + cl));
  return f2(w * (bx - ox / nz_or(oy) * cl), w * (by - cl));
}
// Bipolar (tau, sigma) coordinates (chaos.wgsl:3928-3960, 5107-5145).
VDEV float bip_tau(float2 p) {
  float xp = p.x + 1.0f, xm = p.x - 1.0f, y2 = p.y * p.y;
  return 0.5f * (logf(fmaxf(xp * xp + y2, 1e-30f)) - logf(fmaxf(xm * xm + y2, 1e-30f)));
}
VDEV float bip_sigma(float2 p) { return P_PI - atan2f(p.y, p.x + 1.0f) - atan2f(p.y, 1.0f - p.x); }
VAR(b_mod) {  // P = radius, distance
  float tau = bip_tau(p), sg = bip_sigma(p);
  if (tau < P[0] && -tau < P[0]) {
    float rs = fmaxf(P[0], 1e-30f), tr = 2.0f * rs;
    float arg = tau + rs + P[1] * rs;
    tau = arg - floorf(arg / tr) * tr - rs;
  }
  float t = coshf(tau) - cosf(sg);
  if (fabsf(t) < 1e-30f) t = 1e-30f;
  return f2(w * sinhf(tau) / t, w * sinf(sg) / t);
}
VAR(b_transform) {  // P = rotate, power, move, split
  float pw = fmaxf(1.0f, P[1]);
  float tau = bip_tau(p) / pw + P[2];
  float sg = P_PI - atan2f(p.y, p.x + 1.0f) - atan2f(p.y, 1.0f - p.x) + P[0];
  float k = floorf(RAND01() * pw);
  sg = sg / pw + (2.0f * P_PI / pw) * k;
  tau += p.x >= 0.0f ? P[3] : -P[3];
  float t = coshf(tau) - scos(sg);
  if (fabsf(t) < 1e-30f) t = 1e-30f;
  return f2(w * sinhf(tau) / t, w * ssin(sg) / t);
}
VAR(parallel) {  // P = x1width, x1tilesize, x1mod1, x1mod2, x1height, x1move, x2width, x2tilesize, x2mod1, x2mod2
  if (w == 0.0f) return f2(0.0f, 0.0f);
  const bool first = RAND01() < 0.5f;
  const float wd = first ? P[0] : P[6], ts = first ? P[1] : P[7], m1 = first ? P[2] : P[8];
  const float r1 = fmaxf(first ? P[3] * P[2] : P[9] * P[8], 1e-30f);
  const float ht = first ? P[4] : 0.5f, mv = first ? w * P[5] : -w * 1.0f;
  float x = RAND01() < 0.5f ? wd : -wd;
  float ox = ts * (p.x + wround(x * logf(fmaxf(RAND01(), 1e-30f))));
  float oy;
  if (p.y > m1) {
    float a = p.y + m1;
    oy = ht * (-m1 + (a - floorf(a / r1) * r1)) + mv;
  } else if (p.y < -m1) {
    float a = m1 - p.y;
    oy = ht * (m1 - (a - floorf(a / r1) * r1)) + mv;
  } else {
    oy = ht * p.y + mv;
  }
  return f2(ox, oy);
}
VAR(waves3) {  // P = scalex, scaley, freqx, freqy, sx_freq, sy_freq
  float sx = 0.5f * P[0] * (1.0f + ssin(p.y * P[4])), sy = 0.5f * P[1] * (1.0f + ssin(p.x * P[5]));
  return f2(w * (p.x + ssin(p.y * P[2]) * sx), w * (p.y + ssin(p.x * P[3]) * sy));
}
VAR(waves4) {  // P = scalex, scaley, freqx, freqy, cont, yfact
  float cell = floorf(p.y * P[2] / P_TAU);
  float ax = sinf(cell * 12.9898f + cell * 78.233f + 1.0f + p.y * 0.001f * P[5]) * 43758.5453f;
  ax -= truncf(ax);
  if (P[4] > 0.5f) ax = ax > 0.5f ? 1.0f : 0.0f;
  return f2(w * (p.x + ssin(p.y * P[2]) * ax * ax * P[0]), w * (p.y + ssin(p.x * P[3]) * P[1]));
}
VAR(scry2) {  // P = sides, star, circle
  const i32 kMax = 50;
  i32 sides = min(max(f2i(P[0]), 1), kMax);
  float sa, ca;
  ssincos(P_TAU / (float)sides, &sa, &ca);
  float sins = ssin(-P[1] * P_PI * 0.5f), coss = scos(P[1] * P_PI * 0.5f);
  float sinc = ssin(P[2] * P_PI * 0.5f), cosc = scos(P[2] * P_PI * 0.5f);
  float xr = p.x, yr = p.y;
  float r2 = xr * coss + fabsf(yr) * sins;
  float cr = sqrtf(xr * xr + yr * yr);
  i32 iters = 0;
  for (i32 i = 0; i < kMax && i < sides - 1; ++i) {
    float sw = xr * ca - yr * sa;
    yr = xr * sa + yr * ca;
    xr = sw;
    r2 = fmaxf(r2, xr * coss + fabsf(yr) * sins);
    iters = i + 1;
  }
  r2 = r2 * cosc + cr * sinc;
  float r1 = r2;
  r2 = iters > 1 ? r2 * r2 : fabsf(r2) * r2;
  if (w == 0.0f) return f2(0.0f, 0.0f);
  float d = r1 * (r2 + 1.0f / w);
  if (d == 0.0f) return f2(0.0f, 0.0f);
  return p * (1.0f / d);
}
VAR(ennepers2) {  // P = a, b, c
  float x = p.x, y = p.y, r2 = 1.0f / fmaxf(x * x + y * y, 1e-30f);
  float dxy = (P[0] * x) * (P[0] * x) - (P[1] * y) * (P[1] * y);
  return f2(w * x * (P[0] * P[0] - dxy * r2 - P[2] * sqrtf(fabsf(x))),
            w * y * (P[1] * P[1] - dxy * r2 - P[2] * sqrtf(fabsf(y))));
}
VAR(apollony) {
  const float s3 = 1.7320508075688772f;
  float dx = 1.0f + s3 - p.x;
  float den = fmaxf(dx * dx + p.y * p.y, 1e-30f);
  float a0 = 3.0f * dx / den - (1.0f + s3) / (2.0f + s3), b0 = 3.0f * p.y / den;
  float ab = fmaxf(a0 * a0 + b0 * b0, 1e-30f);
  float fx = a0 / ab, fy = -b0 / ab;
  i32 br = f2i(floorf(4.0f * RAND01())) % 3;
  float x, y;
  if (br == 0) { x = a0; y = b0; }
  else if (br == 1) { x = -fx * 0.5f - fy * s3 * 0.5f; y = fx * s3 * 0.5f - fy * 0.5f; }
  else { x = -fx * 0.5f + fy * s3 * 0.5f; y = -fx * s3 * 0.5f - fy * 0.5f; }
  return f2(w * x, w * y);
}
VAR(circlecrop) {  // P = radius, x, y, scatter_area, zero
  float ca = wclamp(P[3], -1.0f, 1.0f);
  float dx = p.x - P[1], dy = p.y - P[2];
  float rad = sqrtf(dx * dx + dy * dy), ang = atan2f(dy, dx);
  float rdc = P[0] + (RAND01() * 0.5f * ca);
  bool esc = rad > P[0], zero = P[4] > 0.5f;
  if (zero && esc) return f2(0.0f, 0.0f);
  if (esc) return f2(w * rdc * cosf(ang) + P[1], w * rdc * sinf(ang) + P[2]);
  return f2(w * dx + P[1], w * dy + P[2]);
}

// ----------------------------------------------------- complex dynamics
VDEV float2 cpow_int(float2 z, i32 k) {  // binary exponentiation
  float2 r = f2(1.0f, 0.0f), b = z;
  while (k > 0) {
    if (k & 1) r = cmul(r, b);
    b = csqr(b);
    k >>= 1;
  }
  return r;
}
VAR(newton) {  // P = n
  i32 n = min(max(f2i(P[0] + 0.5f), 2), 8);
  float2 zn = cpow_int(p, n), zm = cpow_int(p, n - 1);
  float nf = (float)n, nm1 = (float)(n - 1);
  float2 num = f2(nm1 * zn.x + 1.0f, nm1 * zn.y), den = f2(nf * zm.x, nf * zm.y);
  if (dot2(den, den) < 1.0e-20f) return p * w;
  return w * cdiv(num, den);
}
DCV(newton) {  // nearest root of z^n = 1 after one Newton step
  i32 n = min(max(f2i(P[0] + 0.5f), 2), 8);
  float2 zn = cpow_int(p, n), zm = cpow_int(p, n - 1);
  float nf = (float)n, nm1 = (float)(n - 1);
  float2 num = f2(nm1 * zn.x + 1.0f, nm1 * zn.y), den = f2(nf * zm.x, nf * zm.y);
  float2 z = dot2(den, den) < 1.0e-20f ? p : cdiv(num, den);
  i32 best = 0;
  float bd = 1.0e30f;
  const float step = 6.2831853f / (float)n;
  for (i32 k = 0; k < 8 && k < n; ++k) {
    float ang = step * (float)k;
    float2 d = z - f2(cosf(ang), sinf(ang));
    float d2 = dot2(d, d);
    if (d2 < bd) { bd = d2; best = k; }
  }
  return hsl_rgb((float)best / (float)n, 1.0f, 0.55f);
}
VDEV float2 ship_step(float2 z, float cx, float cy) {
  return csqr(f2(fabsf(z.x), fabsf(z.y))) + f2(cx, cy);
}
VDEV float2 magnet_step(float2 z, float cx, float cy, bool* ok) {
  float2 c0 = f2(cx, cy);
  float2 num = csqr(z) + c0 - f2(1.0f, 0.0f), den = 2.0f * z + c0 - f2(2.0f, 0.0f);
  *ok = dot2(den, den) >= 1.0e-20f;
  return *ok ? csqr(cdiv(num, den)) : z;
}
VDEV float2 nova_step(float2 z, float cx, float cy, float relax, bool* ok) {
  float2 num = cpow_int(z, 3) - f2(1.0f, 0.0f), den = 3.0f * csqr(z);
  *ok = dot2(den, den) >= 1.0e-20f;
  return *ok ? z - relax * cdiv(num, den) + f2(cx, cy) : z;
}
VDEV float2 halley_step(float2 z, float cx, float cy, bool* ok) {
  float2 fz = cpow_int(z, 3) - f2(1.0f, 0.0f), fp = 3.0f * csqr(z), fpp = 6.0f * z;
  float2 num = 2.0f * cmul(fz, fp), den = 2.0f * csqr(fp) - cmul(fz, fpp);
  *ok = dot2(den, den) >= 1.0e-20f;
  return *ok ? z - cdiv(num, den) + f2(cx, cy) : z;
}
VAR(burning_ship) { return w * ship_step(p, P[0], P[1]); }  // P = cx, cy
VAR(magnet1) {
  bool ok;
  float2 z = magnet_step(p, P[0], P[1], &ok);
  return w * z;
}
VAR(nova) {  // P = cx, cy, relax
  bool ok;
  return w * nova_step(p, P[0], P[1], P[2], &ok);
}
VAR(halley) {
  bool ok;
  return w * halley_step(p, P[0], P[1], &ok);
}
// Smooth escape-band colour after up to 12 map iterations (chaos.wgsl:5484).
VDEV float3 escape_band(float2 z, int kind, float cx, float cy, float relax) {
  i32 iters = 0;
  for (i32 i = 0; i < 12; ++i) {
    bool ok = true;
    if (kind == 0) z = ship_step(z, cx, cy);
    else if (kind == 1) z = magnet_step(z, cx, cy, &ok);
    else if (kind == 2) z = nova_step(z, cx, cy, relax, &ok);
    else z = halley_step(z, cx, cy, &ok);
    iters = i + 1;
    if (dot2(z, z) > 256.0f) break;
  }
  float r = fmaxf(len2(z), 1.0001f);
  float mu = (float)iters + 1.0f - log2f(fmaxf(logf(r), 1.0e-6f));
  return hsl_rgb(wfract(mu * 0.12f), 1.0f, 0.55f);
}
DCV(burning_ship) { return escape_band(p, 0, P[0], P[1], 0.0f); }
DCV(magnet1) { return escape_band(p, 1, P[0], P[1], 0.0f); }
DCV(nova) { return escape_band(p, 2, P[0], P[1], P[2]); }
DCV(halley) { return escape_band(p, 3, P[0], P[1], 0.0f); }
VAR(blaschke) {  // P = ax, ay
  float2 a = f2(P[0], P[1]);
  float2 num = cmul(p, p - a), den = f2(1.0f, 0.0f) - cmul(f2(P[0], -P[1]), p);
  if (dot2(den, den) < 1.0e-20f) return p * w;
  return w * cdiv(num, den);
}
VAR(cayley) {  // P = s
  float2 si = f2(0.0f, P[0]), den = p + si;
  if (dot2(den, den) < 1.0e-20f) return p * w;
  return w * cdiv(p - si, den);
}
