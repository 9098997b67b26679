// pyr3-b200 variation library, part 4: indices 154..192 (circus .. lace_js),
// restated from the reference's src/shaders/chaos.wgsl lines 3700-4640.
// Where the reference calls plain sin/cos (angle-bounded or deliberately
// unguarded arguments) this file does too; safe trig elsewhere.
#pragma once

VAR(circus) {  // P = scale
  float s1 = P[0] == 0.0f ? 1e30f : 1.0f / P[0];
  float r = sqrtf(p.x * p.x + p.y * p.y), a = atan2f(p.y, p.x);
  float rs = r <= 1.0f ? r * P[0] : r * s1;
  return f2(w * rs * cosf(a), w * rs * sinf(a));
}
VAR(asteria) {  // P = alpha
  float sa, ca;
  ssincos(P_PI * P[0], &sa, &ca);
  float x0 = w * p.x, y0 = w * p.y;
  float r = x0 * x0 + y0 * y0;
  float xx = (fabsf(x0) - 1.0f) * (fabsf(x0) - 1.0f), yy = (fabsf(y0) - 1.0f) * (fabsf(y0) - 1.0f);
  bool in1 = r < 1.0f;
  bool keep = (in1 && sqrtf(yy + xx) < 1.0f) ? RAND01() > 0.35f : !in1;
  if (keep) return f2(x0, y0);
  float rx = x0 * ca - y0 * sa, ry = x0 * sa + y0 * ca;
  float den = sqrtf(fmaxf(1.0f - ry * ry, 1e-30f));
  float t = -fabsf(ry) + 1.0f;
  float nx = rx / den * (1.0f - sqrtf(fmaxf(1.0f - t * t, 0.0f)));
  return f2(nx * ca + ry * sa, -nx * sa + ry * ca);
}
VAR(clifford_js) {  // P = a, b, c, d
  return f2(w * (ssin(P[0] * p.y) + P[2] * scos(P[0] * p.x)), w * (ssin(P[1] * p.x) + P[3] * scos(P[1] * p.y)));
}
VAR(devil_warp) {  // P = a, b, effect, warp, rmin, rmax
  float x = p.x, y = p.y;
  float r2 = 1.0f / fmaxf(x * x + y * y, 1e-30f);
  float ba = x * x + r2 * P[1] * y * y, bb = y * y + r2 * P[0] * x * x;
  float r = (ba > 0.0f ? wpow(ba, P[3]) : 0.0f) - (bb > 0.0f ? wpow(bb, P[3]) : 0.0f);
  r = P[2] * wclamp(r, P[4], P[5]);
  return f2(x * (1.0f + r), y * (1.0f + r));
}
// Integer lattice noise in [0, 1] (chaos.wgsl:3808), i32 arithmetic wraps.
VDEV float lattice_noise(i32 x) {
  u32 s = ((u32)x << 13) ^ (u32)x;
  u32 r = (s * (s * s * 15731u + 789221u) + 1376312589u) & 0x7fffffffu;
  return (float)r * (float)(1.0 / 2147483647.0);
}
VAR(voron) {  // P = k, step, num, xseed, yseed
  i32 xs = f2i(P[3]), ys = f2i(P[4]);
  float st = P[1] == 0.0f ? 1e-30f : P[1];
  i32 M = f2i(floorf(p.x / st)), N = f2i(floorf(p.y / st));
  float rmin = 20.0f, X0 = 0.0f, Y0 = 0.0f;
  for (i32 i = -1; i < 2; ++i) {
    i32 M1 = M + i;
    for (i32 j = -1; j < 2; ++j) {
      i32 N1 = N + j;
      i32 K = min(max(1 + f2i(floorf(P[2] * lattice_noise(19 * M1 + 257 * N1 + xs))), 1), 26);
      for (i32 l = 0; l < K; ++l) {
        float X = (lattice_noise(l + 64 * M1 + 15 * N1 + xs) + (float)M1) * P[1];
        float Y = (lattice_noise(l + 21 * M1 + 33 * N1 + ys) + (float)N1) * P[1];
        float ox = p.x - X, oy = p.y - Y;
        float r = sqrtf(ox * ox + oy * oy);
        if (r < rmin) { rmin = r; X0 = X; Y0 = Y; }
      }
    }
  }
  return f2(w * (P[0] * (p.x - X0) + X0), w * (P[0] * (p.y - Y0) + Y0));
}
VAR(henon) { return f2(w * (P[2] - P[0] * p.x * p.x + p.y), w * P[1] * p.x); }  // P = a, b, c
VAR(atan) {  // P = mode, stretch
  float nm = w * 2.0f / P_PI;
  i32 mode = f2i(P[0]);
  if (mode == 0) return f2(w * p.x, nm * atanf(P[1] * p.y));
  if (mode == 1) return f2(nm * atanf(P[1] * p.x), w * p.y);
  if (mode == 2) return f2(nm * atanf(P[1] * p.x), nm * atanf(P[1] * p.y));
  return f2(0.0f, 0.0f);
}
VAR(cardioid) {  // P = a
  float th = atan2f(p.y, p.x);
  float r = w * sqrtf(fmaxf(p.x * p.x + p.y * p.y + ssin(P[0] * th) + 1.0f, 0.0f));
  return f2(r * cosf(th), r * sinf(th));
}
VAR(chrysanthemum) {
  float u = 21.0f * P_PI * RAND01();
  float p4 = sinf(17.0f * u / 3.0f);
  float p8 = sinf(2.0f * cosf(3.0f * u) - 28.0f * u);
  float p44 = p4 * p4 * p4 * p4, p82 = p8 * p8;
  float p88 = p82 * p82 * p82 * p82;
  float r = w * 0.1f * (5.0f * (1.0f + sinf(11.0f * u / 5.0f)) - 4.0f * p44 * p88);
  return f2(r * cosf(u), r * sinf(u));
}
VAR(bcollide) {  // P = num, a
  float num = fmaxf(1.0f, P[0]);
  float k_pi = num / P_PI, pi_k = P_PI / num, ak = P_PI * P[1] / num;
  float xp = p.x + 1.0f, xm = p.x - 1.0f, y2 = p.y * p.y;
  float tau = 0.5f * (logf(fmaxf(xp * xp + y2, 1e-30f)) - logf(fmaxf(xm * xm + y2, 1e-30f)));
  float sg = P_PI - atan2f(p.y, xp) - atan2f(p.y, 1.0f - p.x);
  i32 alt = f2i(sg * k_pi);
  float off = (alt & 1) == 0 ? ak : -ak;
  float fold = sg + off - floorf((sg + off) / pi_k) * pi_k;
  float sigma = (float)alt * pi_k + fold;
  float t = coshf(tau) - scos(sigma);
  if (fabsf(t) < 1e-30f) t = 1e-30f;
  return f2(w * sinhf(tau) / t, w * ssin(sigma) / t);
}
VAR(bsplit) {  // P = x, y
  float ax = p.x + P[0];
  float sx = sinf(ax);
  if (fabsf(sx) < 1e-6f) return f2(0.0f, 0.0f);
  float cx = cosf(ax);
  float tx = sx / cx;
  if (fabsf(cx) < 1e-6f) tx = wsign(tx) * 1e6f;
  return f2(w / tx * scos(p.y + P[1]), w / sx * (-1.0f * p.y + P[1]));
}
VAR(bulge) {  // P = n
  float rs = fmaxf(sqrtf(p.x * p.x + p.y * p.y), 1e-30f);
  float k = wpow(rs, P[0]) / rs;
  return f2(w * p.x * k, w * p.y * k);
}
VAR(checks) {  // P = x, y, size, rnd
  float cs = 1.0f / (P[2] + 1e-6f);
  i32 sxy = f2i(wround(p.x * cs)) + f2i(wround(p.y * cs));
  float rnx = P[3] * RAND01();
  float rny = P[3] * RAND01();
  float dx, dy;
  if ((sxy & 1) == 0) { dx = -P[0] + rnx; dy = -P[1]; }
  else { dx = P[0]; dy = P[1] + rny; }
  return f2(w * (p.x + dx), w * (p.y + dy));
}
// fract(sin(k . p + seed) * 43758.5453) amplifies one ulp of the sine by
// 4e4: the argument is separately rounded and the sine is the correctly
// rounded f32 value (double sine rounded once), as the reference's f32 ops.
VDEV float circ_hash(float x, float y, float kx, float ky, float seed) {
  float a = mul_rn(x, kx) + mul_rn(y, ky) + seed;
  float ar = mul_rn((float)sin((double)a), 43758.5453f);
  return ar - truncf(ar);
}
VAR(circular) {  // P = angle, seed
  float ca = P[0] * P_PI / 180.0f;
  float aux = circ_hash(p.x, p.y, 12.9898f, 78.233f, P[1]);
  float rnd = (2.0f * (RAND01() + aux) - 2.0f) * ca;
  float rad = sqrtf(p.x * p.x + p.y * p.y), ang = atan2f(p.y, p.x);
  return f2(w * cosf(ang + rnd) * rad, w * sinf(ang + rnd) * rad);
}
VAR(circular2) {  // P = angle, seed, x, y
  float ca = P[0] * P_PI / 180.0f;
  float aux = circ_hash(p.x, p.y, P[2], P[3], P[1]);
  float rnd = (2.0f * (RAND01() + aux) - 2.0f) * ca;
  float rad = sqrtf(p.x * p.x + p.y * p.y), ang = atan2f(p.y, p.x);
  return f2(w * cosf(ang + rnd) * rad, w * sinf(ang + rnd) * rad);
}
VAR(corners) {  // P = x, y, mult_x, mult_y, x_power, y_power, xy_power_add, log_mode, log_base
  float xs = p.x * p.x, ys = p.y * p.y, ex, ey;
  if (P[7] == 0.0f) {
    ex = wpow(fmaxf(xs, 0.0f), P[4] + P[6]) * P[2];
    ey = wpow(fmaxf(ys, 0.0f), P[5] + P[6]) * P[3];
  } else {
    float lb = logf(fmaxf(fabsf(P[8]), 1.000001f));
    ex = wpow(logf((xs * P[2]) + 3.0f) / lb, P[4] + 2.25f + P[6]) - 1.33f;
    ey = wpow(logf((ys * P[3]) + 3.0f) / lb, P[5] + 2.25f + P[6]) - 1.33f;
  }
  return f2(p.x > 0.0f ? w * ex + P[0] : -w * ex - P[0], p.y > 0.0f ? w * ey + P[1] : -w * ey - P[1]);
}
VAR(circleblur) {
  float rad = sqrtf(RAND01());
  float a = RAND01() * 2.0f * P_PI;
  return f2(w * cosf(a) * rad, w * sinf(a) * rad);
}
VAR(fibonacci2) {  // P = sc, sc2
  const float f5 = 0.447213595f, fl = 0.481211825f;
  float s1, c1, s2, c2;
  ssincos(p.y * fl, &s1, &c1);
  ssincos((p.x * P_PI + p.y * fl) * -1.0f, &s2, &c2);
  float e1 = P[0] * expf(P[1] * (p.x * fl));
  float e2 = P[0] * expf(P[1] * ((p.x * fl - p.y * P_PI) * -1.0f));
  return f2(w * (e1 * c1 - e2 * c2) * f5, w * (e1 * s1 - e2 * s2) * f5);
}
// Hyperbolic {p, q} tiling radius (chaos.wgsl:4152-4200).
VDEV float hypertile_r(float pp, float q, bool form1, float* pa_out) {
  float pa = 2.0f * P_PI / fmaxf(3.0f, pp);
  float qa = 2.0f * P_PI / fmaxf(3.0f, q);
  float cpa = cosf(pa);
  float den = cpa + cosf(qa);
  float r2;
  if (form1) r2 = fabsf(den) > 1e-30f ? (1.0f - cpa) / den + 1.0f : 1.0f;
  else r2 = fabsf(den) > 1e-30f ? 1.0f - (cpa - 1.0f) / den : 1.0f;
  *pa_out = pa;
  return r2 > 0.0f ? 1.0f / sqrtf(fmaxf(r2, 1e-30f)) : 1.0f;
}
VDEV float2 hypertile_mobius(float2 p, float w, float re, float im) {
  float a = p.x + re, b = p.y - im;
  float cc = re * p.x - im * p.y + 1.0f, d = re * p.y + im * p.x;
  float vr = w / fmaxf(cc * cc + d * d, 1e-30f);
  return f2(vr * (a * cc + b * d), vr * (b * cc - a * d));
}
VAR(hypertile) {  // P = p, q, n
  float pa;
  float r = hypertile_r(P[0], P[1], true, &pa);
  float s, co;
  ssincos(P[2] * pa, &s, &co);
  return hypertile_mobius(p, w, r * co, r * s);
}
VAR(hypertile1) {  // P = p, q
  float pa;
  float r = hypertile_r(P[0], P[1], false, &pa);
  float rpa = floorf(RAND01() * 10.0f) * pa;
  return hypertile_mobius(p, w, r * cosf(rpa), r * sinf(rpa));
}
VAR(hypertile2) {  // P = p, q
  float pa;
  float r = hypertile_r(P[0], P[1], false, &pa);
  float a = p.x + r, b = p.y, cc = r * p.x + 1.0f, d = r * p.y;
  float xx = a * cc + b * d, yy = b * cc - a * d;
  float vr = w / fmaxf(cc * cc + d * d, 1e-30f);
  float sa, ca;
  ssincos(floorf(RAND01() * 32767.0f) * pa, &sa, &ca);
  return f2(vr * (xx * ca + yy * sa), vr * (yy * ca - xx * sa));
}
VAR(idisc) {
  float a = P_PI / (sqrtf(p.x * p.x + p.y * p.y) + 1.0f);
  float v = atan2f(p.y, p.x) * w / P_PI;
  return f2(v * cosf(a), v * sinf(a));
}
VAR(hole) {  // P = a, inside
  float al = atan2f(p.y, p.x);
  float dl = wpow(fmaxf(al / P_PI + 1.0f, 1e-30f), P[0]);
  float ss = p.x * p.x + p.y * p.y;
  float r = f2i(P[1]) != 0 ? w * dl / fmaxf(ss + dl, 1e-30f) : w * sqrtf(fmaxf(ss + dl, 0.0f));
  return f2(r * cosf(al), r * sinf(al));
}
VAR(kaleidoscope) {  // P = pull, rotate, line_up, x, y
  const float c45 = 0.5253219888177297f, s45 = 0.8509035245341184f;  // cos(45 rad), sin(45 rad)
  float ox = w * (((P[1] * p.x) * c45 - p.y * s45 + P[2]) + P[3]);
  float oy = p.y > 0.0f ? w * (((P[1] * p.y) * c45 + p.x * s45 + P[0] + P[2]) + P[4])
                        : w * ((P[1] * p.y) * c45 + p.x * s45 - P[0] - P[2]);
  return f2(ox, oy);
}
VAR(layered_spiral) {  // P = radius
  float a = p.x * P[0];
  float t = p.x * p.x + p.y * p.y + 1e-30f;
  float s, co;
  ssincos(t, &s, &co);
  return f2(w * a * co, w * a * s);
}
VAR(linear_t) {  // P = pow_x, pow_y
  return f2(w * (p.x >= 0.0f ? 1.0f : -1.0f) * wpow(fmaxf(fabsf(p.x), 1e-30f), P[0]),
            w * (p.y >= 0.0f ? 1.0f : -1.0f) * wpow(fmaxf(fabsf(p.y), 1e-30f), P[1]));
}
VAR(line) {  // P = delta, phi
  float cd = scos(P[0] * P_PI), sd = ssin(P[0] * P_PI), cp = scos(P[1] * P_PI), sp = ssin(P[1] * P_PI);
  float ux = cd * cp, uy = sd * cp;
  float r = sqrtf(fmaxf(ux * ux + uy * uy + sp * sp, 1e-30f));
  float rn = RAND01() * w;
  return f2(ux / r * rn, uy / r * rn);
}
VAR(ovoid) {  // P = x, y
  float r = w / (p.x * p.x + p.y * p.y + 1e-6f);
  return f2(p.x * r * P[0], p.y * r * P[1]);
}
VAR(phoenix_julia) {  // P = power, dist, x_distort, y_distort
  float pw = P[0] == 0.0f ? 1.0f : P[0];
  float px = p.x * (P[2] + 1.0f), py = p.y * (P[3] + 1.0f);
  float k = floorf(RAND01() * 32768.0f);
  // |a| reaches 1e5 rad: separately rounded products keep its last bit.
  float a = mul_rn(atan2f(py, px), P[1] / pw) + mul_rn(k, 2.0f * P_PI / pw);
  return polar2(w * wpow(fmaxf(p.x * p.x + p.y * p.y, 1e-30f), P[1] / (2.0f * pw)), a);
}
VAR(unpolar) {
  float v = (w / P_PI) * 0.5f, r = expf(p.y);
  float s, co;
  ssincos(p.x, &s, &co);
  return f2(v * r * s, v * r * co);
}
VAR(shredrad) {  // P = n, width
  float wd = wclamp(P[1], -1.0f, 1.0f);
  float al = 2.0f * P_PI / fmaxf(0.001f, P[0]);
  float ang = atan2f(p.y, p.x), rad = sqrtf(p.x * p.x + p.y * p.y);
  float xa = (ang + 3.0f * P_PI + al * 0.5f) / al;
  float za = ((xa - floorf(xa)) * wd + floorf(xa)) * al - P_PI - al * 0.5f * wd;
  float s, co;
  ssincos(za, &s, &co);
  return f2(w * rad * co, w * rad * s);
}
VAR(vogel) {  // P = n, scale
  const float phi = 1.61803398874989f;
  const float k = 2.0f * P_PI / (phi * phi);
  float i = floorf(RAND01() * fmaxf(1.0f, P[0])) + 1.0f;
  float r = w * (sqrtf(p.x * p.x + p.y * p.y) + sqrtf(i));
  float s, co;
  ssincos(i * k, &s, &co);
  return f2(r * (co + P[1] * p.x), r * (s + P[1] * p.y));
}
VAR(yin_yang) {  // P = radius, ang1, ang2, dual_t, outside
  float sa, ca, sb, cb;
  ssincos(P_PI * P[1], &sa, &ca);
  ssincos(P_PI * P[2], &sb, &cb);
  float xx = p.x, yy = p.y, inv = 1.0f, RR = P[0];
  if (xx * xx + yy * yy < 1.0f) {
    float nx = xx * ca - yy * sa, ny = xx * sa + yy * ca;
    if (f2i(P[3]) == 1 && RAND01() > 0.5f) {
      inv = -1.0f;
      RR = 1.0f - P[0];
      nx = xx * cb - yy * sb;
      ny = xx * sb + yy * cb;
    }
    xx = nx;
    yy = ny;
    if (yy > 0.0f) {
      float t = sqrtf(fmaxf(1.0f - yy * yy, 0.0f));
      float k = xx / fmaxf(fabsf(t), 1e-30f) * wsign(t);
      float t1 = (t - 0.5f) * 2.0f;
      float al = (1.0f - k) * 0.5f, be = 1.0f - al;
      float k1 = al * RR + be * 1.0f;
      return f2(w * (t1 * k1 + al * (RR - 1.0f)) * inv, w * sqrtf(fmaxf(1.0f - t1 * t1, 0.0f)) * k1 * inv);
    }
    return f2(w * (xx * (1.0f - RR) + RR) * inv, w * (yy * (1.0f - RR)) * inv);
  }
  if (f2i(P[4]) == 1) return p * w;
  return f2(0.0f, 0.0f);
}
VAR(squish) {  // P = power
  float pw = fmaxf(2.0f, P[0]), ip = 1.0f / pw;
  float ax = fabsf(p.x), ay = fabsf(p.y), s, q;
  if (ax > ay) {
    s = ax;
    q = p.x > 0.0f ? p.y : 4.0f * s - p.y;
  } else {
    s = ay;
    q = p.y > 0.0f ? 2.0f * s - p.x : 6.0f * s + p.x;
  }
  q = ip * (q + 8.0f * s * floorf(pw * RAND01()));
  if (q <= 1.0f * s) return f2(w * s, w * q);
  if (q <= 3.0f * s) return f2(w * (2.0f * s - q), w * s);
  if (q <= 5.0f * s) return f2(-w * s, w * (4.0f * s - q));
  if (q <= 7.0f * s) return f2(-w * (6.0f * s - q), -w * s);
  return f2(w * s, -w * (8.0f * s - q));
}
VAR(target) {  // P = even, odd, size
  float h = 0.5f * P[2];
  float a = atan2f(p.y, p.x), r = sqrtf(p.x * p.x + p.y * p.y);
  float t = logf(fmaxf(r, 1e-30f));
  if (t < 0.0f) t -= h;
  float at = fabsf(t), sz = fmaxf(fabsf(P[2]), 1e-30f);
  t = at - floorf(at / sz) * sz;
  a += t < h ? P[0] : P[1];
  float s, co;
  ssincos(a, &s, &co);
  return f2(r * co * w, r * s * w);
}
VAR(funnel) {  // P = effect
  float cx = scos(p.x), cy = scos(p.y);
  float sx = 1.0f / (fabsf(cx) < 1e-30f ? 1e-30f : cx), sy = 1.0f / (fabsf(cy) < 1e-30f ? 1e-30f : cy);
  float off = P[0] * P_PI;
  return f2(w * stanh(p.x) * (sx + off), w * stanh(p.y) * (sy + off));
}
VAR(holesq) {
  float x = w * p.x, y = w * p.y, fx = fabsf(x), fy = fabsf(y);
  if (fx + fy > 1.0f) return f2(x, y);
  if (fx > fy) return f2(x >= 0.0f ? (x - fy + 1.0f) * 0.5f : (x + fy - 1.0f) * 0.5f, y);
  return f2(x, y >= 0.0f ? (y - fx + 1.0f) * 0.5f : (y + fx - 1.0f) * 0.5f);
}
VAR(hole2) {  // P = a, b, c, d, inside, shape
  float rh = p.x * p.x + p.y * p.y;
  float th = atan2f(p.y, p.x) * P[3];
  float dl = wpow(fmaxf(th / P_PI + 1.0f, 1e-30f), P[0]) * P[2];
  float b = P[1], r1;
  switch (f2i(P[5])) {
    case 0: r1 = sqrtf(fmaxf(rh, 0.0f)) + dl; break;
    case 1: r1 = sqrtf(fmaxf(rh + dl, 0.0f)); break;
    case 2: r1 = sqrtf(fmaxf(rh + ssin(b * th) + dl, 0.0f)); break;
    case 3: r1 = sqrtf(fmaxf(rh + ssin(th) + dl, 0.0f)); break;
    case 4: r1 = sqrtf(fmaxf(rh + th * th - dl + 1.0f, 0.0f)); break;
    case 5: r1 = sqrtf(fmaxf(rh + fabsf(stan(th)) + dl, 0.0f)); break;
    case 6: r1 = sqrtf(fmaxf(rh * (1.0f + ssin(b * th)) + dl, 0.0f)); break;
    case 7: r1 = sqrtf(fmaxf(rh + fabsf(ssin(0.5f * b * th)) + dl, 0.0f)); break;
    case 8: r1 = sqrtf(fmaxf(rh + ssin(P_PI * ssin(b * th)) + dl, 0.0f)); break;
    case 9: r1 = sqrtf(fmaxf(rh + (ssin(b * th) + ssin(2.0f * b * th + P_PI * 0.5f)) * 0.5f + dl, 0.0f)); break;
    default: r1 = 1.0f; break;
  }
  float rf = f2i(P[4]) != 0 ? w / fmaxf(r1, 1e-30f) : w * r1;
  float s, co;
  ssincos(th, &s, &co);
  return f2(rf * co, rf * s);
}
VAR(lace_js) {
  const float r = 2.0f, s32 = 0.8660254037844386f;
  float r0 = sqrtf(p.x * p.x + p.y * p.y);
  float wt = RAND01();
  float th, x, y;
  if (wt > 0.75f) {
    th = atan2f(p.y, p.x - 1.0f);
    y = -r0 * cosf(th) / r + 1.0f;
    x = -r0 * sinf(th) / r;
  } else if (wt > 0.5f) {
    th = atan2f(p.y - s32, p.x + 0.5f);
    y = -r0 * cosf(th) / r - 0.5f;
    x = -r0 * sinf(th) / r + s32;
  } else if (wt > 0.25f) {
    th = atan2f(p.y + s32, p.x + 0.5f);
    y = -r0 * cosf(th) / r - 0.5f;
    x = -r0 * sinf(th) / r - s32;
  } else {
    th = atan2f(p.y, p.x);
    y = -r0 * cosf(th) / r;
    x = -r0 * sinf(th) / r;
  }
  return f2(w * x, w * y);
}
