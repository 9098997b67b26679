// pyr3-b200 variation library, part 7: indices 258..270 (chaotic
// billiards, boosts / lensing / fields, modular forms, Gauss map),
// restated from the reference's src/shaders/chaos.wgsl lines 467-520 and
// 5971-6516.
#pragma once

// Chaotic billiards (chaos.wgsl:5971-6280).  A walker outside the table is
// projected onto its rim, so the ray-circle discriminants below sit next to
// zero and the hit branch turns on their last bit: every product that feeds
// a sum is separately rounded (mul_rn), as the reference's f32 ops are.
// Specular reflection of unit direction v at hit point h with normal n,
// continuing the remaining path length.
VDEV float2 billiard_bounce(float2 h, float vx, float vy, float nx, float ny, float rest) {
  float d = dot_rn(vx, vy, nx, ny);
  float rx = vx - mul_rn(2.0f * d, nx), ry = vy - mul_rn(2.0f * d, ny);
  return f2(h.x + mul_rn(rest, rx), h.y + mul_rn(rest, ry));
}
VAR(billiard_circle) {  // P = radius, step, angle
  float rc = fmaxf(P[0], 1.0e-5f), step = P[1];
  float px = p.x, py = p.y, r0 = len_rn(p.x, p.y);
  if (r0 > rc) {
    px = (px / r0) * rc;
    py = (py / r0) * rc;
    r0 = rc;
  }
  float bx = 1.0f, by = 0.0f;
  if (r0 > 1.0e-6f) { bx = px / r0; by = py / r0; }
  float sa, ca;
  ssincos(P[2], &sa, &ca);
  float vx = mul_rn(bx, ca) - mul_rn(by, sa), vy = mul_rn(bx, sa) + mul_rn(by, ca);
  float dp = dot_rn(px, py, vx, vy);
  float disc = mul_rn(dp, dp) + mul_rn(rc, rc) - dot_rn(px, py, px, py);
  float th = -dp + sqrtf(fmaxf(disc, 0.0f));
  float fx = px + mul_rn(step, vx), fy = py + mul_rn(step, vy);
  if (th > 0.0f && th < step) {
    float2 h = f2(px + mul_rn(th, vx), py + mul_rn(th, vy));
    float2 q = billiard_bounce(h, vx, vy, -h.x / rc, -h.y / rc, step - th);
    fx = q.x;
    fy = q.y;
  }
  return w * f2(fx, fy);
}
VAR(billiard_stadium) {  // P = width, height, step, angle
  const float R = fmaxf(P[1] / 2.0f, 1.0e-5f), w2 = fmaxf(P[0] / 2.0f, 1.0e-5f), step = P[2];
  float px = p.x, py = p.y;
  if (fabsf(px) > w2) {
    float cx = px > 0.0f ? w2 : -w2, dx = px - cx;
    float dist = len_rn(dx, py);
    if (dist > R) {
      px = cx + mul_rn(dx / dist, R);
      py = (py / dist) * R;
    }
  } else if (fabsf(py) > R) {
    py = py > 0.0f ? R : -R;
  }
  float vy, vx;
  ssincos(P[3], &vy, &vx);
  float th = 1.0e10f;
  int wall = 0;
  if (vy > 0.0f) {
    float t = (R - py) / vy, x = px + mul_rn(t, vx);
    if (t >= 0.0f && x >= -w2 && x <= w2 && t < th) { th = t; wall = 1; }
  }
  if (vy < 0.0f) {
    float t = (-R - py) / vy, x = px + mul_rn(t, vx);
    if (t >= 0.0f && x >= -w2 && x <= w2 && t < th) { th = t; wall = 2; }
  }
  for (int side = 0; side < 2; ++side) {  // right then left cap
    float dx = side == 0 ? px - w2 : px + w2;
    float dp = dot_rn(dx, py, vx, vy);
    float disc = mul_rn(dp, dp) + mul_rn(R, R) - dot_rn(dx, py, dx, py);
    if (disc >= 0.0f) {
      float t = -dp + sqrtf(disc), x = px + mul_rn(t, vx);
      bool ok = side == 0 ? x >= w2 - 1.0e-5f : x <= -w2 + 1.0e-5f;
      if (t >= 0.0f && ok && t < th) { th = t; wall = 3 + side; }
    }
  }
  float fx = px + mul_rn(step, vx), fy = py + mul_rn(step, vy);
  if (th > 0.0f && th < step) {
    float2 h = f2(px + mul_rn(th, vx), py + mul_rn(th, vy));
    float nx = 0.0f, ny = 0.0f;
    if (wall == 1) ny = -1.0f;
    else if (wall == 2) ny = 1.0f;
    else if (wall == 3) {
      float rl = fmaxf(len_rn(h.x - w2, h.y), 1.0e-5f);
      nx = -(h.x - w2) / rl;
      ny = -h.y / rl;
    } else if (wall == 4) {
      float rl = fmaxf(len_rn(h.x + w2, h.y), 1.0e-5f);
      nx = -(h.x + w2) / rl;
      ny = -h.y / rl;
    }
    float2 q = billiard_bounce(h, vx, vy, nx, ny, step - th);
    fx = q.x;
    fy = q.y;
  }
  return w * f2(fx, fy);
}
VAR(billiard_sinai) {  // P = length, radius, step, angle
  const float L2 = fmaxf(P[0] / 2.0f, 1.0e-5f), R = fmaxf(P[1], 1.0e-5f), step = P[2];
  float px = p.x, py = p.y;
  if (fabsf(px) > L2) px = px > 0.0f ? L2 : -L2;
  if (fabsf(py) > L2) py = py > 0.0f ? L2 : -L2;
  float r0 = len_rn(px, py);
  if (r0 < R) {
    if (r0 > 1.0e-6f) {
      px = (px / r0) * R;
      py = (py / r0) * R;
    } else {
      float th0 = hash01(__float_as_uint(p.x) ^ __float_as_uint(p.y)) * 6.283185307179586f;
      px = R * cosf(th0);
      py = R * sinf(th0);
    }
  }
  float vy, vx;
  ssincos(P[3], &vy, &vx);
  float th = 1.0e10f;
  int wall = 0;
  if (vx < 0.0f) {
    float t = (-L2 - px) / vx, y = py + mul_rn(t, vy);
    if (t >= 0.0f && y >= -L2 && y <= L2 && t < th) { th = t; wall = 1; }
  }
  if (vx > 0.0f) {
    float t = (L2 - px) / vx, y = py + mul_rn(t, vy);
    if (t >= 0.0f && y >= -L2 && y <= L2 && t < th) { th = t; wall = 2; }
  }
  if (vy < 0.0f) {
    float t = (-L2 - py) / vy, x = px + mul_rn(t, vx);
    if (t >= 0.0f && x >= -L2 && x <= L2 && t < th) { th = t; wall = 3; }
  }
  if (vy > 0.0f) {
    float t = (L2 - py) / vy, x = px + mul_rn(t, vx);
    if (t >= 0.0f && x >= -L2 && x <= L2 && t < th) { th = t; wall = 4; }
  }
  {
    float dp = dot_rn(px, py, vx, vy);
    float disc = mul_rn(dp, dp) - (dot_rn(px, py, px, py) - mul_rn(R, R));
    if (disc >= 0.0f) {
      float t = -dp - sqrtf(disc);
      if (t >= 0.0f && t < th) { th = t; wall = 5; }
    }
  }
  float fx = px + mul_rn(step, vx), fy = py + mul_rn(step, vy);
  if (th > 0.0f && th < step) {
    float2 h = f2(px + mul_rn(th, vx), py + mul_rn(th, vy));
    float nx = 0.0f, ny = 0.0f;
    if (wall == 1) nx = 1.0f;
    else if (wall == 2) nx = -1.0f;
    else if (wall == 3) ny = 1.0f;
    else if (wall == 4) ny = -1.0f;
    else if (wall == 5) { nx = h.x / R; ny = h.y / R; }
    float2 q = billiard_bounce(h, vx, vy, nx, ny, step - th);
    fx = q.x;
    fy = q.y;
  }
  return w * f2(fx, fy);
}
VAR(billiard_polygon) {  // P = sides, radius, step, angle
  const u32 sides = f2u(wclamp(P[0] + 0.5f, 3.0f, 12.0f));
  const float R = fmaxf(P[1], 1.0e-5f), step = P[2];
  const float inr = R * cosf(3.141592653589793f / (float)sides);
  float px = p.x, py = p.y;
  float r0 = len_rn(px, py);
  if (r0 > inr) {
    float s = inr / fmaxf(r0, 1.0e-6f);
    px *= s;
    py *= s;
  }
  float vy, vx;
  ssincos(P[3], &vy, &vx);
  float th = 1.0e10f;
  i32 seg = -1;
  float ax = R * scos(0.0f), ay = R * ssin(0.0f);
  for (u32 k = 0; k < sides; ++k) {
    float ph = (2.0f * 3.141592653589793f * (float)(k + 1u)) / (float)sides;
    float bx = R * scos(ph), by = R * ssin(ph);
    float dx = bx - ax, dy = by - ay;
    float det = mul_rn(-vx, dy) + mul_rn(vy, dx);
    if (fabsf(det) > 1.0e-6f) {
      float t = (mul_rn(-(ax - px), dy) + mul_rn(ay - py, dx)) / det;
      float u = (mul_rn(vx, ay - py) - mul_rn(vy, ax - px)) / det;
      if (t >= 0.0f && u >= 0.0f && u <= 1.0f && t < th) { th = t; seg = (i32)k; }
    }
    ax = bx;
    ay = by;
  }
  float fx = px + mul_rn(step, vx), fy = py + mul_rn(step, vy);
  if (th > 0.0f && th < step && seg != -1) {
    float2 h = f2(px + mul_rn(th, vx), py + mul_rn(th, vy));
    float p0 = (2.0f * 3.141592653589793f * (float)seg) / (float)sides;
    float p1 = (2.0f * 3.141592653589793f * (float)(seg + 1)) / (float)sides;
    float a0x = R * scos(p0), a0y = R * ssin(p0), b0x = R * scos(p1), b0y = R * ssin(p1);
    float ex = b0x - a0x, ey = b0y - a0y;
    float el = fmaxf(len_rn(ex, ey), 1.0e-5f);
    float nx = -ey / el, ny = ex / el;
    if (dot_rn(nx, ny, 0.5f * (a0x + b0x), 0.5f * (a0y + b0y)) > 0.0f) { nx = -nx; ny = -ny; }
    float2 q = billiard_bounce(h, vx, vy, nx, ny, step - th);
    fx = q.x;
    fy = q.y;
  }
  return w * f2(fx, fy);
}
VAR(lorentz_boost) {  // P = rapidity, angle
  float st, ct;
  ssincos(P[1], &st, &ct);
  float rx = p.x * ct + p.y * st, ry = -p.x * st + p.y * ct;
  float ch = coshf(P[0]), sh = sinhf(P[0]);
  float xp = rx * ch + ry * sh, yp = rx * sh + ry * ch;
  return w * f2(xp * ct - yp * st, xp * st + yp * ct);
}
VAR(schwarzschild_lensing) {  // P = mass, eps
  float al = P[0] / (len2(p) + fmaxf(P[1], 1e-6f));
  float sa, ca;
  ssincos(al, &sa, &ca);
  return w * f2(p.x * ca - p.y * sa, p.x * sa + p.y * ca);
}
VAR(field_dipole) {  // P = charge, separation, step, angle
  float d = P[1] * 0.5f;
  float sy, sx;
  ssincos(P[3], &sy, &sx);
  float2 cp = d * f2(sx, sy), cn = -d * f2(sx, sy);
  float2 rp = p - cp, rn = p - cn;
  float dp3 = wpow(dot2(rp, rp) + 1e-4f, 1.5f), dn3 = wpow(dot2(rn, rn) + 1e-4f, 1.5f);
  float2 E = P[0] * (rp / dp3 - rn / dn3);
  return w * (p + P[2] * E);
}
VAR(magnetic_pendulum) {  // P = magnets, radius, strength, damping
  u32 N = f2u(wclamp(P[0], 3.0f, 6.0f));
  float iN = 1.0f / (float)N;
  float2 F = f2(0.0f, 0.0f);
  for (u32 i = 0; i < N; ++i) {
    float s, co;
    ssincos(6.283185307179586f * (float)i * iN, &s, &co);
    float2 r = P[1] * f2(co, s) - p;
    F = F + r / wpow(dot2(r, r) + 1e-4f, 1.5f);
  }
  return w * (p + P[2] * F - P[3] * p);
}
DCV(magnetic_pendulum) {  // nearest magnet's hue
  u32 N = f2u(wclamp(P[0], 3.0f, 6.0f));
  float iN = 1.0f / (float)N, best = 1e30f;
  u32 k = 0u;
  for (u32 i = 0; i < N; ++i) {
    float s, co;
    ssincos(6.283185307179586f * (float)i * iN, &s, &co);
    float2 r = P[1] * f2(co, s) - p;
    float d2 = dot2(r, r);
    if (d2 < best) { best = d2; k = i; }
  }
  return hsl_rgb((float)k * iN, 1.0f, 0.55f);
}

// ---------------------------------------------------------- modular forms
VDEV float2 upper_half(float2 p, float im_floor) {
  return f2(p.x, fmaxf(fabsf(p.y) + fmaxf(im_floor, 0.02f), 0.006435f));
}
VDEV float2 nome(float2 tau) { return cexp(f2(-P_PI * tau.y, P_PI * tau.x)); }
VDEV float2 theta3(float2 q) {  // 1 + 2 sum q^(n^2), 8 terms
  float2 q2 = csqr(q), qn2 = q, odd = cmul(q2, q), sum = qn2;
  for (int n = 2; n <= 8; ++n) {
    qn2 = cmul(qn2, odd);
    sum = sum + qn2;
    odd = cmul(odd, q2);
  }
  return f2(1.0f, 0.0f) + 2.0f * sum;
}
VDEV float2 theta2(float2 q) {  // 2 q^(1/4) sum q^(n(n+1)), 8 terms
  float2 q2 = csqr(q), term = f2(1.0f, 0.0f), ev = q2, sum = term;
  for (int n = 1; n <= 7; ++n) {
    term = cmul(term, ev);
    sum = sum + term;
    ev = cmul(ev, q2);
  }
  return 2.0f * cmul(cpowc(q, f2(0.25f, 0.0f)), sum);
}
VDEV float2 log_squash(float2 z) {  // log(1+|z|) * z/|z| after a +-1e18 clamp
  float2 c0 = f2(wclamp(z.x, -1e18f, 1e18f), wclamp(z.y, -1e18f, 1e18f));
  float m = len2(c0);
  return (logf(1.0f + m) / fmaxf(m, 1e-12f)) * c0;
}
VAR(jacobi_theta) { return w * theta3(nome(upper_half(p, P[0]))); }  // P = im_floor
VDEV float2 lambda_of(float2 q) {
  float2 r2 = csqr(cdiv(theta2(q), theta3(q)));
  return csqr(r2);
}
VAR(modular_lambda) { return w * lambda_of(nome(upper_half(p, P[0]))); }
VAR(klein_j) {
  float2 lam = lambda_of(nome(upper_half(p, P[0])));
  float2 one = f2(1.0f, 0.0f);
  float2 a = one - lam + csqr(lam);
  float2 num = 256.0f * cpow_int(a, 3);
  float2 den = cmul(csqr(lam), csqr(one - lam));
  return w * log_squash(cdiv(num, den));
}
VAR(weierstrass_p) {  // P = omega1_re, omega1_im, omega2_re, omega2_im
  float2 w1 = f2(P[0], P[1]), w2 = f2(P[2], P[3]);
  float2 acc = crecip(csqr(p));
  for (int m = -2; m <= 2; ++m)
    for (int n = -2; n <= 2; ++n) {
      if (m == 0 && n == 0) continue;
      float2 om = (float)m * w1 + (float)n * w2;
      acc = acc + crecip(csqr(p - om)) - crecip(csqr(om));
    }
  return w * log_squash(acc);
}
VDEV float gauss_frac(float t) {
  float r = (t < 0.0f ? -1.0f : 1.0f) / fmaxf(fabsf(t), 1.0e-4f);
  return r - floorf(r);
}
VAR(gauss_map) { return w * f2(gauss_frac(p.x), gauss_frac(p.y)); }
