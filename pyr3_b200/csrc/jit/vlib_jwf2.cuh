// pyr3-b200 variation library, part 3: indices 128..153 (xtrb .. erf),
// restated from the reference's src/shaders/chaos.wgsl lines 2838-3700.
#pragma once

VAR(xtrb) {  // P = power, dist, radius, width, a, b
  const i32 pw = max(1, f2i(P[0]));
  const float pf = (float)pw, radius = P[2], width = P[3];
  const float aB = 0.047f + P[4], aC = 0.047f + P[5], aA = P_PI - aB - aC;
  float sA2, cA2, sB2, cB2, sC2, cC2, sC, cC;
  ssincos(0.5f * aA, &sA2, &cA2);
  ssincos(0.5f * aB, &sB2, &cB2);
  ssincos(0.5f * aC, &sC2, &cC2);
  ssincos(aC, &sC, &cC);
  const float as = radius * (sC2 / cC2 + sB2 / cB2);
  const float bs = radius * (sC2 / cC2 + sA2 / cA2);
  const float cs = radius * (sB2 / cB2 + sA2 / cA2);
  const float w1 = 1.0f - width, w2 = 2.0f * width, w3 = 1.0f - width * width;
  const float S2 = radius * (as + bs + cs);
  const float Ha = S2 / as / 6.0f, Hb = S2 / bs / 6.0f, Hc = S2 / cs / 6.0f;
  const float ab = as / bs, ac = as / cs, ba = bs / as, bc = bs / cs, ca = cs / as, cb = cs / bs;
  const float S2a = 6.0f * Ha, S2b = 6.0f * Hb, S2c = 6.0f * Hc;
  const float S2bc = S2 / (bs + cs) / 6.0f, S2ab = S2 / (as + bs) / 6.0f, S2ac = S2 / (as + cs) / 6.0f;
  const u32 absN = (u32)abs(pw);
  const float cN = P[1] / pf / 2.0f;
  const float U = p.y + radius, V = p.x * sC - p.y * cC + radius;
  const float M = floorf(U / S2a), N = floorf(V / S2b);
  float Al = U - M * S2a, Be = V - N * S2b;
  float Ga = S2c - ac * Al - bc * Be;
  const float R = RAND01();
  const bool neg = Ga <= 0.0f;
  if (neg) {
    Al = S2a - Al;
    Be = S2b - Be;
    Ga = -Ga;
  }
  float A1 = 0.0f, B1 = 0.0f, G1 = 0.0f, D1 = 0.0f;
  const bool thin = R >= w3;
  if (Be < Al) {
    if (Ga < Be) {
      if (thin) { D1 = width * Be; G1 = width * Ga; }
      else { G1 = w1 * Ga + w2 * Hc * Ga / Be; D1 = w1 * Be + w2 * S2ab * (3.0f - Ga / Be); }
      A1 = S2a - ba * D1 - ca * G1;
      B1 = D1;
    } else if (Ga < Al) {
      if (thin) { G1 = width * Ga; D1 = width * Be; }
      else { D1 = w1 * Be + w2 * Hb * Be / Ga; G1 = w1 * Ga + w2 * S2ac * (3.0f - Be / Ga); }
      A1 = S2a - ba * D1 - ca * G1;
      B1 = D1;
    } else {
      if (thin) { A1 = width * Al; B1 = width * Be; }
      else { B1 = w1 * Be + w2 * Hb * Be / Al; A1 = w1 * Al + w2 * S2ac * (3.0f - Be / Al); }
    }
  } else {
    if (Ga < Al) {
      if (thin) { D1 = width * Al; G1 = width * Ga; }
      else { G1 = w1 * Ga + w2 * Hc * Ga / Al; D1 = w1 * Al + w2 * S2ab * (3.0f - Ga / Al); }
      B1 = S2b - ab * D1 - cb * G1;
      A1 = D1;
    } else if (Ga < Be) {
      if (thin) { G1 = width * Ga; D1 = width * Al; }
      else { D1 = w1 * Al + w2 * Ha * Al / Ga; G1 = w1 * Ga + w2 * S2bc * (3.0f - Al / Ga); }
      B1 = S2b - ab * D1 - cb * G1;
      A1 = D1;
    } else {
      if (thin) { B1 = width * Be; A1 = width * Al; }
      else { A1 = w1 * Al + w2 * Ha * Al / Be; B1 = w1 * Be + w2 * S2bc * (3.0f - Al / Be); }
    }
  }
  if (neg) {
    A1 = S2a - A1;
    B1 = S2b - B1;
  }
  A1 += M * S2a;
  B1 += N * S2b;
  const float inx = (B1 - radius + (A1 - radius) * cC) / sC, iny = A1 - radius;
  const float br = RAND01();  // drawn unconditionally (WGSL select evaluates both arms)
  const float bf = (float)(absN > 0u ? f2u(br * (float)absN) : 0u);
  const float ang = (atan2f(iny, inx) + P_TAU * bf) / pf;
  const float rp = wpow(inx * inx + iny * iny, cN);
  float s, co;
  ssincos(ang, &s, &co);
  return f2(w * w * rp * co, w * w * rp * s);
}
VAR(gridout) {
  float x = p.x, y = p.y;
  float rx = x >= 0.0f ? floorf(x + 0.5f) : ceilf(x - 0.5f);
  float ry = y >= 0.0f ? floorf(y + 0.5f) : ceilf(y - 0.5f);
  float dx = 0.0f, dy = 0.0f;
  if (ry <= 0.0f) {
    if (rx > 0.0f) { if (-ry >= rx) dx = 1.0f; else dy = 1.0f; }
    else { if (ry <= rx) dx = 1.0f; else dy = -1.0f; }
  } else {
    if (rx > 0.0f) { if (ry >= rx) dx = -1.0f; else dy = 1.0f; }
    else { if (ry > -rx) dx = -1.0f; else dy = -1.0f; }
  }
  return f2(w * (x + dx), w * (y + dy));
}
VAR(blur_circle) {  // P = hole
  float u0 = RAND01(), u1 = RAND01();
  float x = 2.0f * u0 - 1.0f, y = 2.0f * u1 - 1.0f;
  float ax = fabsf(x), ay = fabsf(y), s = ax > ay ? ax : ay;
  float a = atan2f(y, x);
  const float q3 = 3.0f * P_PI / 4.0f, q1 = P_PI / 4.0f;
  float ps = a < -q3 ? ay : (a < -q1 ? 2.0f * s + x : (a < q1 ? 4.0f * s + y : (a < q3 ? 6.0f * s - x : 8.0f * s - y)));
  return polar2((w * 4.0f / P_PI) * s + P[0], q1 * ps / s - P_PI);
}
VAR(bipolar2) {  // P = shift, a, b, c, d, e, f1, g1, h
  const float hp = P_PI * 0.5f, tp = 2.0f / P_PI;
  float x2y2 = (p.x * p.x + p.y * p.y) * P[7];
  float t = x2y2 + P[1], x2 = P[2] * p.x;
  float y = P[3] * atan2f(P[5] * p.y, x2y2 - P[4]) + (-hp * P[0]);
  if (y > hp) y = -hp + wmod(y + hp, P_PI);
  else if (y < -hp) y = hp - wmod(hp - y, P_PI);
  float fn = t + x2, gn = t - x2;
  if (gn == 0.0f || (fn / gn) <= 0.0f) return f2(0.0f, 0.0f);
  return f2(w * P[6] * tp * logf(fn / gn), w * tp * y * P[8]);
}
VAR(bubble2) {  // P = x, y
  float r = w / (0.25f * sq2(p) + 1.0f);
  return f2(p.x * r * P[0], p.y * r * P[1]);
}
VAR(acosh) {
  float2 d = csqrt(csqr(p) - f2(1.0f, 0.0f));
  float2 z = clog(p + d) * (w * 2.0f / P_PI);
  return RAND01() >= 0.5f ? -z : z;
}
VAR(arcsinh) { return clog(p + csqrt(csqr(p) + f2(1.0f, 0.0f))) * (w * 2.0f / P_PI); }
VAR(arctanh) { return clog(cdiv(p + f2(1.0f, 0.0f), f2(1.0f, 0.0f) - p)) * (w * 2.0f / P_PI); }
VAR(acoth) {
  float2 rz = crecip(p);
  float2 h = 0.5f * clog(cdiv(rz + f2(1.0f, 0.0f), f2(1.0f, 0.0f) - rz));
  return f2(h.y, h.x) * (w * 2.0f / P_PI);
}
VAR(acosech) {
  float2 rz = crecip(p);
  float2 l = clog(rz + csqrt(csqr(rz) - f2(1.0f, 0.0f)));
  float2 z = f2(l.y, l.x) * (w * 2.0f / P_PI);
  return RAND01() >= 0.5f ? -z : z;
}
VAR(arcsech2) {
  float2 z = crecip(p);
  float2 l = clog(z + cmul(csqrt(z + f2(1.0f, 0.0f)), csqrt(z - f2(1.0f, 0.0f)))) * (w * 2.0f / P_PI);
  return l.y < 0.0f ? f2(l.x, l.y + 1.0f) : f2(-l.x, l.y - 1.0f);
}
VAR(cell2) {  // P = size, a, space_north_x, space_north_y, space_south_x, space_south_y
  float sz = fabsf(P[0]) < 1e-30f ? 1e-30f : P[0];
  float inv = P[1] / sz;
  float cx = floorf(p.x * inv), cy = floorf(p.y * inv);
  float dx = p.x - cx * sz, dy = p.y - cy * sz;
  float sx, sy;
  if (cy >= 0.0f) { sy = cy * P[3]; sx = cx * P[2]; }
  else { sy = -P[5] * cy; sx = cx * P[4]; }
  return f2(w * (dx + sx * sz), -w * (dy + sy * sz));
}
VAR(curl_sp) {  // P = pow, c1, c2, sx, sy
  float pw = P[0] == 0.0f ? 1e-30f : P[0];
  float x = wpow(fabsf(p.x), pw) * wsign(p.x), y = wpow(fabsf(p.y), pw) * wsign(p.y);
  float sa = P[1] * x + P[2] * (x * x - y * y);
  float re = sqrtf(sa * sa + P[3] * P[3]) * (sa > 0.0f ? 1.0f : -1.0f) + 1.0f;
  float sb = P[1] * y + (2.0f * P[2]) * x * y;
  float im = sqrtf(sb * sb + P[4] * P[4]) * (sb > 0.0f ? 1.0f : -1.0f);
  float r = w / fmaxf(wpow(fabsf(re * re + im * im), 1.0f / pw), 1e-30f);
  return f2((x * re + y * im) * r, (y * re - x * im) * r);
}
VAR(murl2) {  // P = c, power
  float sp = P[1] == 0.0f ? 1e-30f : P[1];
  float ip = 1.0f / sp, c1 = P[0] + 1.0f;
  float vp = w * wpow(fabsf(c1), 2.0f * ip) * (c1 >= 0.0f ? 1.0f : -1.0f);
  float a1 = atan2f(p.y, p.x) * sp;
  float r0 = P[0] * wpow(fabsf(sq2(p)), P[1] * 0.5f);
  float s1, c1s;
  ssincos(a1, &s1, &c1s);
  float re0 = r0 * c1s + 1.0f, im0 = r0 * s1;
  float r1 = wpow(fabsf(re0 * re0 + im0 * im0), ip);
  float a2 = atan2f(im0, re0) * 2.0f * ip;
  float s2, c2;
  ssincos(a2, &s2, &c2);
  float re1 = r1 * c2, im1 = r1 * s2;
  float rl = vp / fmaxf(r1 * r1, 1e-30f);
  return f2(rl * (p.x * re1 + p.y * im1), rl * (p.y * re1 - p.x * im1));
}
VAR(lissajous) {  // P = tmin, tmax, a, b, c, d, e
  float t = (P[1] - P[0]) * RAND01() + P[0];
  float yj = RAND01() - 0.5f;
  float drift = P[4] * t + P[6] * yj;
  return f2(w * (ssin(P[2] * t + P[5]) + drift), w * (ssin(P[3] * t) + drift));
}
VAR(spirograph) {  // P = a, b, d, tmin, tmax, ymin, ymax, c1, c2
  float t = (P[4] - P[3]) * RAND01() + P[3];
  float yj = (P[6] - P[5]) * RAND01() + P[5];
  float ab = P[0] + P[1];
  float ratio = ab / (fabsf(P[1]) < 1e-30f ? 1e-30f : P[1]);
  float st, ct;
  ssincos(t, &st, &ct);
  float x1 = ab * ct - P[7] * scos(ratio * t);
  float y1 = ab * st - P[8] * ssin(ratio * t);
  return f2(w * (x1 + P[2] * ct + yj), w * (y1 + P[2] * st + yj));
}
VAR(waffle) {  // P = slices, xthickness, ythickness, rotation
  const float sl = fmaxf(1.0f, floorf(fabsf(P[0]))), inv = 1.0f / sl;
  float sr, cr;
  ssincos(P[3], &sr, &cr);
  const float vc = w * cr, vs = w * sr;
  const u32 mode = f2u(fminf(4.0f, floorf(RAND01() * 5.0f)));
  float a, r;
  if (mode == 0u) {
    float k0 = floorf(RAND01() * sl);
    a = (k0 + RAND01() * P[1]) * inv;
    float k1 = floorf(RAND01() * sl);
    r = (k1 + RAND01() * P[2]) * inv;
  } else if (mode == 1u) {
    float k0 = floorf(RAND01() * sl);
    a = (k0 + RAND01()) * inv;
    r = (floorf(RAND01() * sl) + P[2]) * inv;
  } else if (mode == 2u) {
    a = (floorf(RAND01() * sl) + P[1]) * inv;
    float k1 = floorf(RAND01() * sl);
    r = (k1 + RAND01()) * inv;
  } else if (mode == 3u) {
    a = RAND01();
    float k1 = floorf(RAND01() * sl);
    r = (k1 + P[2] + RAND01() * (1.0f - P[2])) * inv;
  } else {
    float k0 = floorf(RAND01() * sl);
    a = (k0 + P[1] + RAND01() * (1.0f - P[1])) * inv;
    r = RAND01();
  }
  return f2(vc * a + vs * r, -vs * a + vc * r);
}
VDEV float2 glynn_ring(Ctx& c, float r1, float th, float x1, float y1, float w) {
  float ri = r1 * (th + (1.0f - th) * RAND01());
  float ph = P_TAU * RAND01();
  float s, co;
  ssincos(ph, &s, &co);
  return f2(w * (ri * co + x1), w * (ri * s + y1));
}
VAR(glynnSim1) {  // P = radius, radius1, phi1, thickness, pow, contrast
  float s1, c1;
  ssincos(P[2] * (P_PI / 180.0f), &s1, &c1);
  float x1 = P[0] * c1, y1 = P[0] * s1;
  float r = sqrtf(sq2(p));
  if (r < P[0]) return glynn_ring(c, P[1], P[3], x1, y1, w);
  float al = P[0] / fmaxf(r, 1e-30f);
  float x = p.x, y = p.y;
  if (!(RAND01() > P[5] * wpow(fabsf(al), fabsf(P[4])))) {
    x = al * al * p.x;
    y = al * al * p.y;
  }
  float dx = x - x1, dy = y - y1;
  if (dx * dx + dy * dy < P[1] * P[1]) return glynn_ring(c, P[1], P[3], x1, y1, w);
  return f2(w * x, w * y);
}
VAR(glynnSim2) {  // P = radius, thickness, contrast, pow, phi1, phi2
  float p10 = P[4] * (P_PI / 180.0f), p20 = P[5] * (P_PI / 180.0f);
  float rt = P[0] + P[1];
  float gam = P[1] * (2.0f * P[0] + P[1]) / fmaxf(rt, 1e-30f);
  float r = sqrtf(sq2(p));
  if (r < P[0]) {
    float ri = rt - gam * RAND01();
    float ph = p10 + (p20 - p10) * RAND01();
    float s, co;
    ssincos(ph, &s, &co);
    return f2(w * (ri * co), w * (ri * s));
  }
  float al = P[0] / fmaxf(r, 1e-30f);
  if (RAND01() > P[2] * wpow(fabsf(al), fabsf(P[3]))) return p * w;
  return f2(w * (al * al * p.x), w * (al * al * p.y));
}
VAR(glynnSim3) {  // P = radius, thickness, contrast, pow
  float r1 = P[0] + P[1];
  float r2 = (P[0] * P[0]) / fmaxf(r1, 1e-30f);
  float gam = r1 / fmaxf(r1 + r2, 1e-30f);
  float r = sqrtf(sq2(p));
  if (r < r1) {
    float ph = P_TAU * RAND01();
    float ri = RAND01() < gam ? r1 : r2;
    float s, co;
    ssincos(ph, &s, &co);
    return f2(w * (ri * co), w * (ri * s));
  }
  float al = P[0] / fmaxf(r, 1e-30f);
  if (RAND01() > P[2] * wpow(fabsf(al), fabsf(P[3]))) return p * w;
  return f2(w * (al * al * p.x), w * (al * al * p.y));
}
VAR(flipy) { return f2(w * p.x, w * p.y * (p.x > 0.0f ? -1.0f : 1.0f)); }
VAR(eclipse) {  // P = shift
  if (fabsf(p.y) <= w) {
    float c2 = sqrtf(fmaxf(w * w - p.y * p.y, 0.0f));
    float ox = w * p.x;
    if (fabsf(p.x) <= c2) {
      float xs = p.x + P[0] * w;
      ox = fabsf(xs) >= c2 ? -w * p.x : w * xs;
    }
    return f2(ox, w * p.y);
  }
  return p * w;
}
VAR(barycentroid) {  // P = a, b, c, d
  float d00 = P[0] * P[0] + P[1] * P[1], d01 = P[0] * P[2] + P[1] * P[3];
  float d02 = P[0] * p.x + P[1] * p.y, d11 = P[2] * P[2] + P[3] * P[3], d12 = P[2] * p.x + P[3] * p.y;
  float den = d00 * d11 - d01 * d01;
  if (fabsf(den) < 1e-30f) return p * w;
  float id = 1.0f / den;
  float u = (d11 * d02 - d01 * d12) * id, v = (d00 * d12 - d01 * d02) * id;
  return f2(w * (sqrtf(u * u + p.x * p.x) * wsign(u)), w * (sqrtf(v * v + p.y * p.y) * wsign(v)));
}
VAR(chunk) {  // P = a, b, c, d, e, f, mode
  float r = (w * P[0]) * p.x * p.x + (w * P[1]) * p.x * p.y + (w * P[2]) * p.y * p.y +
            (w * P[3]) * p.x + (w * P[4]) * p.y + w * P[5];
  i32 mode = f2i(P[6]);
  if (mode == 0 && r <= 0.0f) return p;
  if (mode == 1 && r > 0.0f) return p;
  return f2(0.0f, 0.0f);
}
VAR(ennepers) {
  float x = p.x, y = p.y;
  return f2(w * (x - (x * x * x) / 3.0f) + x * y * y, w * (y - (y * y * y) / 3.0f) + y * x * x);
}
// Abramowitz & Stegun 7.1.26 rational approximation of erf.
VDEV float erf_as(float x) {
  float s = x >= 0.0f ? 1.0f : -1.0f, ax = fabsf(x);
  float t = 1.0f / (1.0f + 0.3275911f * ax);
  float poly = (((((1.061405429f * t) + -1.453152027f) * t + 1.421413741f) * t + -0.284496736f) * t +
                0.254829592f) * t;
  return s * (1.0f - poly * expf(-ax * ax));
}
VAR(erf) { return f2(w * erf_as(p.x), w * erf_as(p.y)); }
