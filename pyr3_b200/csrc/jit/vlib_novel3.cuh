// pyr3-b200 variation library, part 8: indices 271..309 and 314..325
// (special functions, number-theoretic and bit-pattern warps, optics,
// distributions, wavelets, orbits, attractor maps), restated from the
// reference's src/shaders/chaos.wgsl lines 6518-7715.
#pragma once

// ------------------------------------------------------------ value noise
VDEV float vn_corner(i32 ix, i32 iy) {
  return hash01(((u32)ix * 0x9e3779b1u) ^ ((u32)iy * 0x85ebca77u)) * 2.0f - 1.0f;
}
VDEV float value_noise(float px, float py, i32 period) {  // period <= 0: not periodic
  float fx = floorf(px), fy = floorf(py);
  i32 ix = f2i(fx), iy = f2i(fy);
  float tx = px - fx, ty = py - fy;
  float ux = tx * tx * (3.0f - 2.0f * tx), uy = ty * ty * (3.0f - 2.0f * ty);
  i32 x0 = ix, x1 = ix + 1;
  if (period > 0) {
    i32 m0 = imod(ix, period), m1 = imod(ix + 1, period);
    x0 = m0 < 0 ? m0 + period : m0;
    x1 = m1 < 0 ? m1 + period : m1;
  }
  float b = wmix(vn_corner(x0, iy), vn_corner(x1, iy), ux);
  float t = wmix(vn_corner(x0, iy + 1), vn_corner(x1, iy + 1), ux);
  return wmix(b, t, uy);
}
VDEV float lich_field(float2 p, float freq, float br, float radial, i32 oct) {
  float r = len2(p), ang = atan2f(p.y, p.x) / P_TAU;
  float u = wmix(p.x * freq, (ang + 0.5f) * br, radial);
  float v = wmix(p.y * freq, r * freq, radial);
  i32 period = max(f2i(wround(br)), 1);
  float sum = 0.0f, amp = 1.0f, tot = 0.0f;
  for (i32 k = 0; k < oct; ++k) {
    sum += amp * value_noise(u, v, period);
    tot += amp;
    amp *= 0.5f;
    u *= 2.0f;
    v *= 2.0f;
    period *= 2;
  }
  return sum / tot;
}

// ------------------------------------------------------ special functions
VDEV float bessel_j0f(float x) {  // Abramowitz & Stegun 9.4.1 / 9.4.3
  float ax = fabsf(x);
  if (ax < 3.0f) {
    float y = (x * x) / 9.0f;
    return 1.0f + y * (-2.2499997f + y * (1.2656208f + y * (-0.3163866f + y * (0.0444479f +
                  y * (-0.0039444f + y * 0.0002100f)))));
  }
  float z = 3.0f / ax, y = z * z;
  float amp = 0.79788456f + y * (-0.00000077f + y * (-0.00552740f + y * (-0.00009512f +
              y * (0.00137237f + y * (-0.00072805f + y * 0.00014476f)))));
  float ph = ax - 0.78539816f + y * (-0.04166397f + y * (-0.00003954f + y * (0.00262573f +
             y * (-0.00054125f + y * (-0.00029333f + y * 0.00013558f)))));
  return (amp / sqrtf(ax)) * scos(ph);
}
VDEV float airy_ai(float x) {  // asymptotic tails, Maclaurin series in the middle
  if (x > 4.0f) {
    float xi = (2.0f / 3.0f) * wpow(x, 1.5f);
    return expf(-xi) / (2.0f * 1.7724539f * wpow(x, 0.25f));
  }
  if (x < -5.0f) {
    float ax = -x, xi = (2.0f / 3.0f) * wpow(ax, 1.5f);
    return ssin(xi + 0.78539816f) / (1.7724539f * wpow(ax, 0.25f));
  }
  float x3 = x * x * x, f = 1.0f, tf = 1.0f, g = x, tg = x;
  for (int k = 1; k < 12; ++k) {
    float kf = (float)k;
    tf *= x3 / ((3.0f * kf - 1.0f) * (3.0f * kf));
    f += tf;
    tg *= x3 / ((3.0f * kf) * (3.0f * kf + 1.0f));
    g += tg;
  }
  return 0.355028053887817f * f - 0.258819403792807f * g;
}
VDEV float struve_h1f(float xin) {  // power series, 16 terms
  float h = 0.5f * wclamp(xin, -10.0f, 10.0f), h2 = h * h;
  float term = h2 / (0.8862269f * 1.3293404f), sum = term;
  for (int m = 1; m < 16; ++m) {
    float mf = (float)m;
    term = term * (-h2) / ((mf + 0.5f) * (mf + 1.5f));
    sum += term;
  }
  return sum;
}
VDEV float erfinv_w(float xin) {  // Winitzki's closed-form approximation, a = 0.147
  float x = wclamp(xin, -0.999999f, 0.999999f);
  const float a = 0.147f;
  float l1 = logf(1.0f - x * x);
  float t1 = 2.0f / (P_PI * a) + 0.5f * l1;
  float in = sqrtf(fmaxf(t1 * t1 - l1 / a, 0.0f)) - t1;
  return wsign(x) * sqrtf(fmaxf(in, 0.0f));
}
VDEV float ell_E(float m) {  // Hastings polynomial approximations
  float m1 = wclamp(1.0f - m, 0.0f, 1.0f), l = logf(1.0f / fmaxf(m1, 1.0e-6f));
  return (1.0f + m1 * (0.4630151f + m1 * 0.1077812f)) + (m1 * (0.2452727f + m1 * 0.0412496f)) * l;
}
VDEV float ell_K(float m) {
  float m1 = wclamp(1.0f - m, 1.0e-3f, 1.0f), l = logf(1.0f / m1);
  return (1.3862944f + m1 * (0.1119723f + m1 * 0.0725296f)) + (0.5f + m1 * (0.1213478f + m1 * 0.0288729f)) * l;
}
VDEV float cheb_t(float x, i32 n) {
  if (n <= 0) return 1.0f;
  if (n == 1) return x;
  float a = 1.0f, b = x, t = x;
  for (i32 k = 2; k <= n; ++k) { t = 2.0f * x * b - a; a = b; b = t; }
  return t;
}
VDEV float legendre_p(float x, i32 n) {
  if (n <= 0) return 1.0f;
  if (n == 1) return x;
  float a = 1.0f, b = x, t = x;
  for (i32 k = 1; k < n; ++k) {
    float fk = (float)k;
    t = ((2.0f * fk + 1.0f) * x * b - fk * a) / (fk + 1.0f);
    a = b;
    b = t;
  }
  return t;
}
VDEV float assoc_legendre(i32 l, i32 m, float u) {
  float pmm = 1.0f;
  if (m > 0) {
    float s = sqrtf(fmaxf(1.0f - u * u, 0.0f)), fact = 1.0f;
    for (i32 i = 1; i <= m; ++i) { pmm = pmm * (-fact) * s; fact += 2.0f; }
  }
  if (l == m) return pmm;
  float pm1 = u * (2.0f * (float)m + 1.0f) * pmm;
  if (l == m + 1) return pm1;
  float pll = 0.0f;
  for (i32 ll = m + 2; ll <= l; ++ll) {
    float fl = (float)ll;
    pll = ((2.0f * fl - 1.0f) * u * pm1 - (fl + (float)m - 1.0f) * pmm) / (fl - (float)m);
    pmm = pm1;
    pm1 = pll;
  }
  return pll;
}
VDEV float sph_y(float th, i32 l, i32 m) {
  i32 mm = abs(m);
  return wclamp(fabsf(assoc_legendre(l, mm, scos(th)) * scos((float)mm * th)), 0.0f, 4.0f);
}
VDEV float laguerre(i32 k, float al, float x) {
  if (k <= 0) return 1.0f;
  float a = 1.0f, b = 1.0f + al - x;
  if (k == 1) return b;
  for (i32 j = 1; j < k; ++j) {
    float fj = (float)j;
    float c = ((2.0f * fj + 1.0f + al - x) * b - (fj + al) * a) / (fj + 1.0f);
    a = b;
    b = c;
  }
  return b;
}
VDEV float radial_psi2(i32 n, i32 l, float rho) {
  float r = fmaxf(rho, 0.0f);
  float lg = laguerre(n - l - 1, 2.0f * (float)l + 1.0f, r);
  float rp = 1.0f;
  for (i32 j = 0; j < 2 * l; ++j) rp *= r;
  return rp * expf(-r) * (lg * lg);
}

// --------------------------------------------------- fixed-point lattices
VDEV u32 bmask(u32 bits) { return (1u << bits) - 1u; }
VDEV u32 fp_enc(float c, float ext, u32 bits) {
  float s = fmaxf(ext, 1.0e-4f), n = (c + s) / (2.0f * s);
  return min(f2u((n - floorf(n)) * (float)(1u << bits)), bmask(bits));
}
VDEV float fp_dec(u32 i, float ext, u32 bits) {
  float s = fmaxf(ext, 1.0e-4f);
  return (((float)i + 0.5f) / (float)(1u << bits)) * 2.0f * s - s;
}
VDEV u32 pow3u(u32 n) {
  u32 p = 1u;
  for (u32 i = 0; i < n; ++i) p *= 3u;
  return p;
}
VDEV u32 tri_enc(float c, float ext, u32 trits) {
  float s = fmaxf(ext, 1.0e-4f);
  u32 cells = pow3u(trits);
  float n = (c + s) / (2.0f * s);
  return min(f2u((n - floorf(n)) * (float)cells), cells - 1u);
}
VDEV float tri_dec(u32 i, float ext, u32 trits) {
  float s = fmaxf(ext, 1.0e-4f);
  return (((float)i + 0.5f) / (float)pow3u(trits)) * 2.0f * s - s;
}
VDEV u32 peano_scr(u32 idx, u32 trits) {
  bool flip = false;
  u32 out = 0u;
  for (u32 k = trits; k > 0u; --k) {
    u32 place = pow3u(k - 1u);
    u32 d = (idx / place) % 3u;
    u32 e = flip ? 2u - d : d;
    out += e * place;
    if (e & 1u) flip = !flip;
  }
  return out;
}
VDEV u32 rev_bits(u32 x, u32 bits) {
  u32 r = 0u;
  for (u32 k = 0; k < bits; ++k) { r = (r << 1) | (x & 1u); x >>= 1; }
  return r;
}
VDEV u32 spread_bits(u32 x, u32 bits) {
  u32 r = 0u;
  for (u32 i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (i << 1);
  return r;
}

// ----------------------------------------------------------- variations
VAR(nbody_lensing) {  // P = c1x, c1y, c2x, c2y, m1, m2, g, eps
  float e = fmaxf(P[7], 5.0e-3f);
  float2 d1 = f2(P[0], P[1]) - p, d2 = f2(P[2], P[3]) - p;
  float r1 = dot2(d1, d1) + e, r2 = dot2(d2, d2) + e;
  float2 disp = (P[6] * P[4] / (r1 * sqrtf(r1))) * d1;
  disp = disp + (P[6] * P[5] / (r2 * sqrtf(r2))) * d2;
  return w * (p + disp);
}
VAR(curl_noise) {  // P = freq, amp
  float f = fmaxf(P[0], 1.0e-3f), sx = p.x * f, sy = p.y * f;
  const float h = 1.0e-2f;
  float dx = (value_noise(sx + h, sy, 0) - value_noise(sx - h, sy, 0)) / (2.0f * h);
  float dy = (value_noise(sx, sy + h, 0) - value_noise(sx, sy - h, 0)) / (2.0f * h);
  return w * (p + P[1] * f2(wclamp(dy, -8.0f, 8.0f), wclamp(-dx, -8.0f, 8.0f)));
}
VAR(bessel_j0) { return w * (bessel_j0f(P[0] * len2(p)) * p); }  // P = freq
VAR(airy_radial) { return w * ((3.0f * airy_ai(P[0] * (len2(p) - P[1]))) * p); }  // P = scale, shift
VAR(cornu_spiral) {  // P = freq
  float t = P[0] * p.x, s = fabsf(t), sg = t < 0.0f ? -1.0f : 1.0f;
  float f = (1.0f + 0.926f * s) / (2.0f + 1.792f * s + 3.104f * (s * s));
  float g = 1.0f / (2.0f + 4.142f * s + 3.492f * (s * s) + 6.670f * (s * s * s));
  float sa, ca;
  ssincos((P_PI * (s * s)) / 2.0f, &sa, &ca);
  return w * f2(sg * (0.5f + f * sa - g * ca), sg * (0.5f - f * ca - g * sa) + 0.25f * p.y);
}
VAR(struve_h1) { return w * ((0.6f * struve_h1f(P[0] * len2(p))) * p); }  // P = freq
VAR(radical_inverse) {  // P = extent, bits
  u32 b = f2u(wclamp(P[1], 2.0f, 24.0f));
  u32 rx = rev_bits(fp_enc(p.x, P[0], b), b) & bmask(b), ry = rev_bits(fp_enc(p.y, P[0], b), b) & bmask(b);
  return w * f2(fp_dec(rx, P[0], b), fp_dec(ry, P[0], b));
}
VAR(gray_code) {  // P = extent, bits
  u32 b = f2u(wclamp(P[1], 2.0f, 24.0f)), m = bmask(b);
  u32 ix = fp_enc(p.x, P[0], b), iy = fp_enc(p.y, P[0], b);
  return w * f2(fp_dec((ix ^ (ix >> 1)) & m, P[0], b), fp_dec((iy ^ (iy >> 1)) & m, P[0], b));
}
VAR(morton_zorder) {  // P = extent, bits
  u32 b = f2u(wclamp(P[1], 2.0f, 16.0f)), m = bmask(b);
  u32 code = spread_bits(fp_enc(p.x, P[0], b), b) | (spread_bits(fp_enc(p.y, P[0], b), b) << 1);
  return w * f2(fp_dec(code & m, P[0], b), fp_dec((code >> b) & m, P[0], b));
}
VAR(chebyshev) {  // P = order_x, order_y
  i32 nx = f2i(wclamp(wround(P[0]), 0.0f, 12.0f)), ny = f2i(wclamp(wround(P[1]), 0.0f, 12.0f));
  return w * f2(cheb_t(wclamp(p.x, -1.0f, 1.0f), nx), cheb_t(wclamp(p.y, -1.0f, 1.0f), ny));
}
VAR(legendre) {  // P = order_x, order_y
  i32 nx = f2i(wclamp(wround(P[0]), 0.0f, 12.0f)), ny = f2i(wclamp(wround(P[1]), 0.0f, 12.0f));
  return w * f2(legendre_p(wclamp(p.x, -1.0f, 1.0f), nx), legendre_p(wclamp(p.y, -1.0f, 1.0f), ny));
}
VAR(spherical_harmonic) {  // P = degree_l, order_m, amount
  float r = len2(p);
  if (r < 1.0e-6f) return f2(0.0f, 0.0f);
  i32 l = f2i(wclamp(wround(P[0]), 0.0f, 6.0f));
  i32 m = f2i(wclamp(wround(P[1]), 0.0f, (float)l));
  float amt = wclamp(P[2], 0.0f, 2.0f);
  float rp = r * wclamp((1.0f - amt) + amt * sph_y(atan2f(p.y, p.x), l, m), -3.0f, 3.0f);
  float ir = 1.0f / r;
  return w * f2(p.x * ir * rp, p.y * ir * rp);
}
VAR(fourier_warp) {  // P = harmonics, amp, phase_seed
  float r = len2(p);
  if (r < 1.0e-6f) return f2(0.0f, 0.0f);
  float th = atan2f(p.y, p.x);
  i32 n = f2i(wclamp(wround(P[0]), 1.0f, 8.0f));
  float amt = wclamp(P[1], 0.0f, 0.9f);
  u32 sb = f2u(wclamp(P[2], 0.0f, 1024.0f));
  float acc = 0.0f;
  for (i32 k = 1; k <= n; ++k) {
    float fk = (float)k;
    float ph = hash01(sb * 2654435761u + (u32)k * 40503u) * P_TAU;
    acc += scos(fk * th + ph) / fk;
  }
  float rp = r * wclamp(1.0f + amt * acc, 0.05f, 3.0f);
  float ir = 1.0f / r;
  return w * f2(p.x * ir * rp, p.y * ir * rp);
}
VAR(snell_refraction) {  // P = n_ratio, strength
  float r = len2(p);
  if (r < 1.0e-6f) return p * w;
  float dx = p.x / r, dy = p.y / r;
  float s2 = wclamp(P[0], 0.05f, 5.0f) * dx, ox, oy;
  if (fabsf(s2) >= 1.0f) {
    ox = dx;
    oy = -dy;
  } else {
    float c2 = sqrtf(fmaxf(1.0f - s2 * s2, 0.0f));
    ox = s2;
    oy = dy >= 0.0f ? c2 : -c2;
  }
  float s = wclamp(P[1], 0.0f, 1.0f);
  float bx = wmix(dx, ox, s), by = wmix(dy, oy, s);
  float bl = fmaxf(len2(f2(bx, by)), 1.0e-6f);
  return (w * r) * f2(bx / bl, by / bl);
}
VAR(grin_lens) {  // P = focal, eps
  float f = fmaxf(fabsf(P[0]), 0.05f), e = fmaxf(fabsf(P[1]), 1.0e-3f);
  float r = len2(p);
  if (r < 1.0e-6f) return p * w;
  float pull = (r / f) * ((e * e) / (r * r + e * e));
  float nr = fmaxf(r - pull, -r);
  return (w * nr) * f2(p.x / r, p.y / r);
}
VAR(caustic_fold) {  // P = freq, amp, phase
  float k = wclamp(P[0], 0.0f, 16.0f), a = wclamp(P[1], 0.0f, 2.0f);
  return w * f2(wclamp(p.x + a * -ssin(k * p.x + P[2]), -8.0f, 8.0f),
                wclamp(p.y + a * -ssin(k * p.y + P[2]), -8.0f, 8.0f));
}
VAR(chladni) {  // P = n, m, step
  float n = wclamp(floorf(P[0] + 0.5f), 1.0f, 12.0f), m = wclamp(floorf(P[1] + 0.5f), 1.0f, 12.0f);
  float an = P_PI * n, am = P_PI * m;
  float cnx = scos(an * p.x), snx = ssin(an * p.x), cmy = scos(am * p.y), smy = ssin(am * p.y);
  float cmx = scos(am * p.x), smx = ssin(am * p.x), cny = scos(an * p.y), sny = ssin(an * p.y);
  float F = cnx * cmy - cmx * cny;
  float gx = -an * snx * cmy + am * smx * cny, gy = -am * cnx * smy + an * cmx * sny;
  float s = F < 0.0f ? -1.0f : 1.0f;
  gx *= s;
  gy *= s;
  float inv = 1.0f / (sqrtf(gx * gx + gy * gy) + 1.0e-4f);
  return w * f2(p.x - P[2] * gx * inv, p.y - P[2] * gy * inv);
}
VAR(standing_wave) {  // P = modes, freq, amp, decay
  float kmax = wclamp(floorf(P[0] + 0.5f), 1.0f, 4.0f), d = wclamp(P[3], 0.0f, 0.999f);
  float dx = 0.0f, dy = 0.0f, ak = P[2];
  for (int k = 1; k <= 4; ++k) {
    float kf = (float)k * P_PI * P[1];
    float gate = (float)k <= kmax ? 1.0f : 0.0f;
    dx += gate * ak * ssin(kf * p.x) * ssin(kf * p.y);
    dy += gate * ak * ssin(kf * p.y) * scos(kf * p.x);
    ak *= d;
  }
  return w * f2(p.x + dx, p.y + dy);
}
VAR(moire) {  // P = freq, beat, angle, amp
  float sa, ca;
  ssincos(P[2], &sa, &ca);
  float u = p.x * ca + p.y * sa, v = -p.x * sa + p.y * ca;
  float f1 = P[0], fb = P[0] + P[1];
  float gx = ssin(f1 * P_PI * p.x) * ssin(fb * P_PI * u);
  float gy = ssin(f1 * P_PI * p.y) * ssin(fb * P_PI * v);
  return w * f2(p.x + P[3] * gx, p.y + P[3] * gy);
}
VDEV float2 shell_out(float2 p, float w, float amp) {
  float r = len2(p);
  float2 dir = r > 1.0e-6f ? p / r : f2(1.0f, 0.0f);
  return (w * (1.5f * (amp / (1.0f + amp)))) * dir;
}
VAR(radial_shell) {  // P = n, l, shell_scale
  i32 n = min(max(f2i(wround(P[0])), 1), 4), l = min(max(f2i(wround(P[1])), 0), n - 1);
  float rho = (2.0f * len2(p)) / ((float)n * fmaxf(P[2], 1.0e-3f));
  return shell_out(p, w, radial_psi2(n, l, rho));
}
VAR(hydrogen_orbital) {  // P = n, l, m, shell_scale, lobe_mix
  i32 n = min(max(f2i(wround(P[0])), 1), 4), l = min(max(f2i(wround(P[1])), 0), n - 1);
  i32 m = min(max(f2i(wround(P[2])), -l), l);
  float rho = (2.0f * len2(p)) / ((float)n * fmaxf(P[3], 1.0e-3f));
  float rad = radial_psi2(n, l, rho);
  float yl = sph_y(atan2f(p.y, p.x), l, m);
  return shell_out(p, w, wmix(rad, rad * (yl * yl), wclamp(P[4], 0.0f, 1.0f)));
}
// Radial CDF-warp helpers: u = r^2 / (1 + r^2) clamped; direction p/r.
VDEV float cdf_u(float2 p) {
  float r2 = dot2(p, p);
  return wclamp(r2 / (1.0f + r2), 1.0e-4f, 1.0f - 1.0e-4f);
}
VDEV float2 cdf_dir(float2 p) {
  float r = sqrtf(dot2(p, p));
  return r < 1.0e-9f ? f2(0.0f, 0.0f) : p / fmaxf(r, 1.0e-12f);
}
VAR(weibull_cdf) {  // P = lambda, k
  float rp = P[0] * wpow(-logf(1.0f - cdf_u(p)), 1.0f / fmaxf(fabsf(P[1]), 0.05f));
  return (w * rp) * cdf_dir(p);
}
VAR(logistic_cdf) {  // P = mu, s
  float u = cdf_u(p);
  float rp = fmaxf(P[0] + P[1] * wclamp(logf(u / (1.0f - u)), -12.0f, 12.0f), 0.0f);
  return (w * rp) * cdf_dir(p);
}
VAR(cauchy_cdf) {  // P = gamma, tail_clamp
  float cap = fmaxf(P[1], 0.01f);
  float rp = wclamp(P[0] * stan(P_PI * (cdf_u(p) - 0.5f)), -cap, cap);
  return (w * rp) * cdf_dir(p);
}
VAR(pareto_cdf) {  // P = x_m, alpha, tail_clamp
  float rp = fminf(P[0] * wpow(1.0f - cdf_u(p), -1.0f / fmaxf(fabsf(P[1]), 0.05f)), fmaxf(P[2], 0.01f));
  return (w * rp) * cdf_dir(p);
}
VAR(morlet) {  // P = freq, sigma, amp
  float r = len2(p), t = r / fmaxf(P[1], 0.05f);
  float psi = expf(-0.5f * fminf(t * t, 80.0f)) * scos(P[0] * r);
  return (w * (1.0f + P[2] * psi)) * p;
}
VAR(mexican_hat) {  // P = sigma, amp
  float t = len2(p) / fmaxf(P[0], 0.05f), t2 = fminf(t * t, 80.0f);
  return (w * (1.0f + P[1] * ((1.0f - t2) * expf(-0.5f * t2)))) * p;
}
VAR(chirp) {  // P = alpha, amp, decay
  float r2 = dot2(p, p);
  float psi = expf(-P[2] * fminf(r2, 160.0f)) * ssin(P[0] * r2);
  return (w * (1.0f + P[1] * psi)) * p;
}
VAR(kepler_orbit) {  // P = e, scale
  float e = wclamp(P[0], 0.0f, 0.95f), M = atan2f(p.y, p.x);
  float a = P[1] * (len2(p) + 1.0e-6f), E = M;
  for (int k = 0; k < 2; ++k) {
    float s, c0;
    ssincos(E, &s, &c0);
    E = E - (E - e * s - M) / fmaxf(1.0f - e * c0, 0.05f);
  }
  float se, ce;
  ssincos(E, &se, &ce);
  return w * f2(a * (ce - e), a * sqrtf(fmaxf(1.0f - e * e, 0.0f)) * se);
}
VAR(restricted_3body) {  // P = mu, step, coriolis
  float mu = wclamp(P[0], 0.01f, 0.5f);
  float2 r1 = p - f2(-mu, 0.0f), r2 = p - f2(1.0f - mu, 0.0f);
  float d1 = wpow(dot2(r1, r1) + 1.0e-3f, 1.5f), d2 = wpow(dot2(r2, r2) + 1.0e-3f, 1.5f);
  float2 g = p - (1.0f - mu) * (r1 / d1) - mu * (r2 / d2);
  float2 disp = P[1] * (g + P[2] * f2(-g.y, g.x));
  float dl = len2(disp);
  if (dl > 2.0f) disp = disp * (2.0f / dl);
  return w * (p + disp);
}
VAR(hill_epicyclic) {  // P = kappa, phase, shear
  float k = wclamp(P[0], 0.2f, 2.0f);
  float sf, cf;
  ssincos(P[1] * k, &sf, &cf);
  return w * f2(p.x * cf - (sf / k) * p.y, ((2.0f * k) * sf * p.x + p.y * cf) + P[2] * p.x);
}
VAR(torus_knot) {  // P = p, q, radius, tube
  float ph = atan2f(p.y, p.x);
  float pf = fmaxf(wround(P[0]), 1.0f), qf = fmaxf(wround(P[1]), 1.0f);
  float rr = P[2] + (P[3] * wclamp(len2(p), 0.0f, 1.0f)) * scos(qf * ph);
  float s, co;
  ssincos(pf * ph, &s, &co);
  return w * f2(rr * co, rr * s);
}
VAR(braid_warp) {  // P = strands, twist, crossings
  float n = fmaxf(wround(P[0]), 2.0f), cr = fmaxf(wround(P[2]), 1.0f);
  float r = len2(p), th = atan2f(p.y, p.x);
  float a = (th + P_PI) / P_TAU, lane = floorf(a * n), fr = a * n - lane;
  float sg = (f2i(lane) & 1) == 1 ? -1.0f : 1.0f;
  float dth = P[1] * sg * ssin(P_PI * fr) * ssin(cr * P_PI * fr) * wclamp(r, 0.0f, 1.0f);
  float s, co;
  ssincos(th + dth, &s, &co);
  return (w * r) * f2(co, s);
}
VAR(airy_caustic) {  // P = scale, r0, amp
  float env = wclamp(1.0f + P[2] * airy_ai(P[0] * (len2(p) - P[1])), 0.05f, 3.0f);
  return w * (env * p);
}
VAR(elliptic_E) {  // P = scale
  float r2 = dot2(p, p);
  return w * (P[0] * ell_E(r2 / (1.0f + r2))) * cdf_dir(p);
}
VAR(elliptic_K) {  // P = scale, tail_clamp
  float r2 = dot2(p, p);
  float rp = fminf(P[0] * ell_K(r2 / (1.0f + r2)), fmaxf(P[1], 0.01f));
  return (w * rp) * cdf_dir(p);
}
VAR(gaussian_cdf) {  // P = mu, sigma
  float rp = fmaxf(P[0] + P[1] * 1.4142135f * erfinv_w(2.0f * cdf_u(p) - 1.0f), 0.0f);
  return (w * rp) * cdf_dir(p);
}
VAR(levy_cdf) {  // P = c, tail_clamp
  float e = erfinv_w(1.0f - cdf_u(p));
  float rp = fminf(fmaxf(P[0], 1.0e-4f) / fmaxf(2.0f * e * e, 1.0e-6f), fmaxf(P[1], 0.01f));
  return (w * rp) * cdf_dir(p);
}
VAR(peano) {  // P = extent, trits
  u32 t = f2u(wclamp(P[1], 2.0f, 15.0f));
  u32 sx = peano_scr(tri_enc(p.x, P[0], t), t), sy = peano_scr(tri_enc(p.y, P[0], t), t);
  return w * f2(tri_dec(sx, P[0], t), tri_dec(sy, P[0], t));
}
VAR(lichtenberg) {  // P = freq, branches, radial, detail, strength
  const float H = 1.0e-2f;
  float freq = fmaxf(P[0], 1.0e-3f), br = wclamp(wround(P[1]), 1.0f, 16.0f);
  float rad = wclamp(P[2], 0.0f, 1.0f);
  i32 oct = f2i(wclamp(wround(P[3]), 1.0f, 4.0f));
  float st = fmaxf(P[4], 0.0f);
  if (len2(p) < 1.0e-4f) return p * w;
  float f0 = lich_field(p, freq, br, rad, oct);
  float gx = (lich_field(p + f2(H, 0.0f), freq, br, rad, oct) - lich_field(p - f2(H, 0.0f), freq, br, rad, oct)) / (2.0f * H);
  float gy = (lich_field(p + f2(0.0f, H), freq, br, rad, oct) - lich_field(p - f2(0.0f, H), freq, br, rad, oct)) / (2.0f * H);
  float g2 = fmaxf(gx * gx + gy * gy, 1.0e-3f);
  float2 step = -(f0 / g2) * f2(gx, gy);
  float sl = len2(step);
  if (sl > 2.0f) step = step * (2.0f / sl);
  return w * (p + st * step);
}
VDEV float sigmoid(float t) { return 1.0f / (1.0f + expf(-t)); }
VAR(copula_gaussian) {  // P = strength, rho
  float s = fmaxf(P[0], 1.0e-3f);
  float u = wclamp(sigmoid(s * p.x), 1.0e-4f, 1.0f - 1.0e-4f), v = wclamp(sigmoid(s * p.y), 1.0e-4f, 1.0f - 1.0e-4f);
  float zx = 1.4142135f * erfinv_w(2.0f * u - 1.0f), zy = 1.4142135f * erfinv_w(2.0f * v - 1.0f);
  float rho = wclamp(P[1], -0.95f, 0.95f);
  return w * f2(p.x, (rho * zx + sqrtf(fmaxf(1.0f - rho * rho, 0.0f)) * zy) / s);
}
VAR(copula_clayton) {  // P = strength, theta
  float s = fmaxf(P[0], 1.0e-3f);
  float u = wclamp(sigmoid(s * p.x), 1.0e-4f, 1.0f - 1.0e-4f), v = wclamp(sigmoid(s * p.y), 1.0e-4f, 1.0f - 1.0e-4f);
  float th = wclamp(P[1], 0.05f, 8.0f);
  float base = fmaxf(wpow(u, -th) + wpow(v, -th) - 1.0f, 1.0e-6f);
  float up = wclamp(wpow(u, -th - 1.0f) * wpow(base, -1.0f - 1.0f / th), 1.0e-4f, 1.0f - 1.0e-4f);
  return w * f2(p.x, wclamp(logf(up / (1.0f - up)), -12.0f, 12.0f) / s);
}
VAR(schwarz_christoffel) {  // P = sides
  float n = fmaxf(wround(P[0]), 3.0f);
  i32 ni = f2i(n);
  float r = len2(p);
  float2 z = r > 0.999f ? p * (0.999f / fmaxf(r, 1.0e-12f)) : p;
  float a = 2.0f / n, coef = 1.0f;
  float2 acc = f2(0.0f, 0.0f);
  for (i32 k = 0; k < 10; ++k) {
    i32 pi = ni * k + 1;
    acc = acc + (coef / (float)pi) * cpow_int(z, pi);
    coef = coef * (a + (float)k) / (float)(k + 1);
  }
  return w * acc;
}
VAR(doyle) {  // P = p, q
  float pp = fmaxf(fabsf(P[0]), 1.0f);
  float2 L = clog(p);
  float pitch = P[1] / pp;
  float us = L.x + pitch * L.y;
  float rip = 0.12f * (ssin(pp * L.y) + scos(pp * L.y - P_TAU * us));
  return w * cexp(f2(us + rip, L.y + pitch * rip));
}
VAR(quasicrystal) {  // P = symmetry, freq
  i32 n = f2i(wclamp(wround(P[0]), 2.0f, 12.0f));
  float freq = fmaxf(P[1], 1.0e-3f);
  float2 g = f2(0.0f, 0.0f);
  for (i32 k = 0; k < n; ++k) {
    float th = P_PI * (float)k / (float)n;
    float2 dir = f2(cosf(th), sinf(th));
    g = g - ssin(freq * dot2(p, dir)) * dir;
  }
  g = g / (float)n;
  return w * (p + 0.4f * g);
}
VAR(penrose) {  // P = scale, offset
  float sc = fmaxf(P[0], 1.0e-3f);
  float2 v = f2(0.0f, 0.0f);
  for (int j = 0; j < 5; ++j) {
    float th = P_TAU * (float)j / 5.0f;
    float2 dir = f2(cosf(th), sinf(th));
    v = v + floorf(sc * dot2(p, dir) + P[1]) * dir;
  }
  return w * v / sc;
}
VAR(collatz) {  // P = scale, shift
  float sc = fmaxf(fabsf(P[0]), 1.0e-3f);
  float2 z = f2(p.x * sc + P[1], p.y * sc);
  float2 arg = z * (P_PI * 0.5f);
  float2 sn = csin(arg), cs = csin(arg + f2(P_PI * 0.5f, 0.0f));
  float2 even = cmul(0.5f * z, cmul(cs, cs));
  float2 odd = cmul(0.5f * (3.0f * z + f2(1.0f, 0.0f)), cmul(sn, sn));
  return w * (even + odd);
}
VAR(digamma) {  // P = scale, shift; recurrence to z+6 then asymptotic series
  float sc = fmaxf(fabsf(P[0]), 1.0e-3f);
  float2 z = f2(p.x * sc + P[1], p.y * sc);
  float2 sum = f2(0.0f, 0.0f);
  for (int k = 0; k < 6; ++k) {
    sum = sum + crecip(z);
    z = z + f2(1.0f, 0.0f);
  }
  float2 zi = crecip(z), zi2 = cmul(zi, zi), zi4 = cmul(zi2, zi2);
  float2 psi = clog(z) - 0.5f * zi - (1.0f / 12.0f) * zi2 + (1.0f / 120.0f) * zi4;
  return w * (psi - sum);
}
VAR(sprott_poly) {  // P = a1..a5, b1..b5
  float x = p.x, y = p.y, x2 = x * x, xy = x * y, y2 = y * y;
  return w * f2(P[0] * x + P[1] * x2 + P[2] * xy + P[3] * y + P[4] * y2,
                P[5] * x + P[6] * x2 + P[7] * xy + P[8] * y + P[9] * y2);
}
VAR(hopalong) {  // P = a, b, c
  return w * f2(p.y - wsign(p.x) * sqrtf(fabsf(P[1] * p.x - P[2])), P[0] - p.x);
}
VDEV float gm_g(float x, float a) { return a * x + 2.0f * (1.0f - a) * x * x / (1.0f + x * x); }
VAR(gumowski_mira) {  // P = a, b
  float xp = P[1] * p.y + gm_g(p.x, P[0]);
  return w * f2(xp, -p.x + gm_g(xp, P[0]));
}
