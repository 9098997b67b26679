/*
 * pyr3 oracle -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C CPU restatement of the reference (MattAltermatt/pyr3) algorithms
 * on the chaos-game -> histogram -> density-estimation -> tonemap path that
 * run on the reference's HOST (TypeScript) or that the tests need in
 * isolation.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline may load this library, and only as the checker: the product
 * (pyr3_b200/, libpyr3cuda.so) never links or calls it.
 *
 * Parity pins: the ISAAC functions are checked against the reference's
 * tests/fixtures/isaac/golden.json (byte-exact); the pick table against the
 * split rules of src/chaos-xform-pick.test.ts; calibration / DE LUT /
 * spatial kernel against src/calibration.test.ts, src/density.test.ts and
 * src/spatial-filter.test.ts invariants.
 *
 * Every function cites the reference file:line range it restates.  Float
 * work that the reference does on the GPU in f32 (splat, density,
 * visualize) is done here in f32 in the same operation order; host work
 * the reference does in JS doubles (pick table, calibration, LUTs) is done
 * in double.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ ISAAC */
/* src/isaac.ts:17-19 -- RANDSIZL=4, 36 u32 per stream. */
typedef struct {
    uint32_t cnt, a, b, c;
    uint32_t mem[16];
    uint32_t rsl[16];
} or_isaac;

/* src/isaac.ts:35-100 (isaacRound) == chaos.wgsl:243-295 (isaac_round). */
OR_EXPORT void or_isaac_round(or_isaac *s) {
    uint32_t a = s->a;
    s->c += 1u;
    uint32_t b = s->b + s->c;
    uint32_t *mm = s->mem, *r = s->rsl;
    for (int half = 0; half < 2; ++half) {
        int m0 = half * 8, m2 = half ? 0 : 8;
        for (int k = 0; k < 8; ++k) {
            uint32_t mixed;
            switch (k & 3) {
                case 0: mixed = a ^ (a << 13); break;
                case 1: mixed = a ^ (a >> 6); break;
                case 2: mixed = a ^ (a << 2); break;
                default: mixed = a ^ (a >> 16); break;
            }
            uint32_t x = mm[m0 + k];
            a = mixed + mm[m2 + k];
            uint32_t y = mm[(x >> 2) & 15u] + a + b;
            mm[m0 + k] = y;
            b = mm[(y >> 6) & 15u] + x;
            r[m0 + k] = b;
        }
    }
    s->a = a;
    s->b = b;
}

/* src/isaac.ts:103-116 (isaacMix). */
static void or_isaac_mix(uint32_t v[8]) {
    uint32_t a = v[0], b = v[1], c = v[2], d = v[3], e = v[4], f = v[5], g = v[6], h = v[7];
    a ^= b << 11; d += a; b += c;
    b ^= c >> 2;  e += b; c += d;
    c ^= d << 8;  f += c; d += e;
    d ^= e >> 16; g += d; e += f;
    e ^= f << 10; h += e; f += g;
    f ^= g >> 4;  a += f; g += h;
    g ^= h << 8;  b += g; h += a;
    h ^= a >> 9;  c += h; a += b;
    v[0] = a; v[1] = b; v[2] = c; v[3] = d; v[4] = e; v[5] = f; v[6] = g; v[7] = h;
}

/* src/isaac.ts:124-160 (irandinit). */
OR_EXPORT void or_irandinit(or_isaac *s, int seed_from_rsl) {
    uint32_t v[8];
    s->a = s->b = s->c = 0;
    for (int j = 0; j < 8; ++j) v[j] = 0x9e3779b9u;
    for (int i = 0; i < 4; ++i) or_isaac_mix(v);
    if (seed_from_rsl) {
        for (int pass = 0; pass < 2; ++pass) {
            const uint32_t *src = pass == 0 ? s->rsl : s->mem;
            for (int i = 0; i < 16; i += 8) {
                for (int j = 0; j < 8; ++j) v[j] += src[i + j];
                or_isaac_mix(v);
                for (int j = 0; j < 8; ++j) s->mem[i + j] = v[j];
            }
        }
    } else {
        for (int i = 0; i < 16; i += 8) {
            or_isaac_mix(v);
            for (int j = 0; j < 8; ++j) s->mem[i + j] = v[j];
        }
    }
    or_isaac_round(s);
    s->cnt = 16;
}

/* src/isaac.ts:171-179 == chaos.wgsl:297-307 (isaac_irand). */
OR_EXPORT uint32_t or_isaac_irand(or_isaac *s) {
    if (s->cnt == 0) {
        or_isaac_round(s);
        s->cnt = 15;
    } else {
        s->cnt -= 1;
    }
    return s->rsl[s->cnt];
}

/* chaos.wgsl:319-323 (rand01) -- f32(u & 0x0fffffff) * (1/268435455). */
OR_EXPORT float or_rand01(or_isaac *s) {
    uint32_t m = or_isaac_irand(s) & 0x0fffffffu;
    return (float)m * (float)(1.0 / 268435455.0);
}

/* chaos.wgsl:327-331 (rand_11). */
OR_EXPORT float or_rand_11(or_isaac *s) {
    int32_t m = (int32_t)(or_isaac_irand(s) & 0x0fffffffu);
    return (float)(m - 0x07ffffff) * (float)(1.0 / 134217727.0);
}

/* JS ToUint32 of an integral double (ECMA-262 7.1.7) for the walker hash. */
static uint32_t js_to_u32(double d) {
    double m = fmod(trunc(d), 4294967296.0);
    if (m < 0) m += 4294967296.0;
    return (uint32_t)m;
}

/* src/isaac.ts:194-229 (packIsaacStates): PCG32 seeding of randrsl, then
 * irandinit(flag=1).  Output: walkers x 36 u32 in the reference layout
 * [cnt, a, b, c, mem[16], rsl[16]]. */
OR_EXPORT void or_pack_isaac_states(uint32_t walkers, uint32_t seed, uint32_t walker_base,
                                    uint32_t *out) {
    or_isaac st;
    for (uint32_t i = 0; i < walkers; ++i) {
        uint32_t w = walker_base + i;
        /* `w * 2654435761 + 1` is evaluated in JS doubles before ToUint32. */
        uint32_t pcg = seed ^ js_to_u32((double)w * 2654435761.0 + 1.0);
        for (int k = 0; k < 4; ++k) pcg = pcg * 747796405u + 2891336453u;
        for (int k = 0; k < 16; ++k) {
            uint32_t s = pcg;
            pcg = pcg * 747796405u + 2891336453u;
            uint32_t shift = (s >> 28) + 4u;
            uint32_t word = ((s >> shift) ^ s) * 277803737u;
            st.rsl[k] = (word >> 22) ^ word;
        }
        memset(st.mem, 0, sizeof st.mem);
        or_irandinit(&st, 1);
        uint32_t *o = out + (size_t)i * 36;
        o[0] = st.cnt; o[1] = st.a; o[2] = st.b; o[3] = st.c;
        memcpy(o + 4, st.mem, 64);
        memcpy(o + 20, st.rsl, 64);
    }
}

/* ------------------------------------------------------------ pick table */
/* src/genome.ts:482-534 (packXformDistrib).  Rows 0..n-1 are "previous
 * xform = i"; row n is the no-prior-xform fallback.  xaos is n*n row-major
 * (xaos[prev*n + next], 1.0 where the genome omits an entry) or NULL.
 * Returns 0, or -1 on a negative / non-finite product (the reference throws). */
OR_EXPORT int or_pack_xform_distrib(int n, const double *weights, const double *xaos,
                                    uint32_t *rows) {
    const int GRAIN = 16384;
    for (int row = 0; row <= n; ++row) {
        int xi = row < n ? row : -1;
        uint32_t *out = rows + (size_t)row * GRAIN;
        double sum = 0.0;
        for (int i = 0; i < n; ++i) {
            double m = (xi >= 0 && xaos) ? xaos[xi * n + i] : 1.0;
            double d = weights[i] * m;
            if (!isfinite(d) || d < 0) return -1;
            sum += d;
        }
        memset(out, 0, sizeof(uint32_t) * GRAIN);
        if (sum == 0.0) continue;
        double dr = sum / GRAIN;
        int j = 0;
        double t = weights[0] * ((xi >= 0 && xaos) ? xaos[xi * n + 0] : 1.0);
        double r = 0.0;
        for (int i = 0; i < GRAIN; ++i) {
            while (r >= t) {
                ++j;
                double m = (xi >= 0 && xaos && j < n) ? xaos[xi * n + j] : 1.0;
                t += (j < n ? weights[j] : 0.0) * m;
                if (j > n + 1) break; /* unreachable for finite sums; bounds the scan */
            }
            out[i] = (uint32_t)j;
            r += dr;
        }
    }
    return 0;
}

/* --------------------------------------------------------------- palette */
/* src/palette.ts:52-58 (catmullRom, B = 0.5). */
static double or_catmull(double u, double xa, double xb, double xc, double xd) {
    const double B = 0.5;
    double c = u * u * u * (-B * xa + (2 - B) * xb + (B - 2) * xc + B * xd);
    c += u * u * (2 * B * xa + (B - 3) * xb + (3 - 2 * B) * xc - B * xd);
    c += u * (-B * xa + B * xc);
    return c + xb;
}

static double clamp01d(double v) { return v < 0 ? 0 : (v > 1 ? 1 : v); }

/* src/palette.ts:71-125 (bakeLUT) without hue rotation.  Stops must be
 * sorted by t (the reference sorts; callers here pass them sorted).
 * mode: 0 = linear, 1 = step, 2 = smooth.  out = 256 x RGBA f32, alpha 0. */
OR_EXPORT void or_bake_lut(int ns, const double *st, const double *sr, const double *sg,
                           const double *sb, int mode, float *out) {
    for (int i = 0; i < 256; ++i) {
        double t = i / 255.0;
        int lo = 0, hi = ns - 1;
        for (int s = 0; s < ns - 1; ++s) {
            if (t >= st[s] && t <= st[s + 1]) { lo = s; hi = s + 1; break; }
        }
        double r, g, b;
        if (mode == 1) {
            r = sr[lo]; g = sg[lo]; b = sb[lo];
        } else {
            double span = st[hi] - st[lo];
            if (span == 0) span = 1;
            double u = clamp01d((t - st[lo]) / span);
            if (mode == 2 && ns >= 3) {
                int a = lo - 1 < 0 ? 0 : lo - 1;
                int d = hi + 1 > ns - 1 ? ns - 1 : hi + 1;
                r = clamp01d(or_catmull(u, sr[a], sr[lo], sr[hi], sr[d]));
                g = clamp01d(or_catmull(u, sg[a], sg[lo], sg[hi], sg[d]));
                b = clamp01d(or_catmull(u, sb[a], sb[lo], sb[hi], sb[d]));
            } else {
                r = sr[lo] + (sr[hi] - sr[lo]) * u;
                g = sg[lo] + (sg[hi] - sg[lo]) * u;
                b = sb[lo] + (sb[hi] - sb[lo]) * u;
            }
        }
        out[i * 4 + 0] = (float)r;
        out[i * 4 + 1] = (float)g;
        out[i * 4 + 2] = (float)b;
        out[i * 4 + 3] = 0.0f;
    }
}

/* ------------------------------------------------- calibration and LUTs */
/* src/calibration.ts:37-43 (deriveCalibration). */
OR_EXPORT void or_derive_calibration(double scale, double samples, double brightness, int os,
                                     double *k1, double *k2) {
    double os2 = (double)os * (double)os;
    *k1 = (brightness * 255.0 * 268.0) / 256.0;
    *k2 = (os2 * scale * scale) / (255.0 * samples);
}

/* src/density.ts:78-99 (buildKernelNormLut): 257 entries, double sums
 * rounded to f32. */
OR_EXPORT void or_kernel_norm_lut(float *out) {
    for (int r = 0; r <= 256; ++r) {
        if (r == 0) { out[0] = 1.0f; continue; }
        double sigma = r / 3.0;
        double inv2s2 = 1.0 / (2.0 * sigma * sigma);
        double r2 = (double)r * r, sum = 0.0;
        for (int dy = -r; dy <= r; ++dy)
            for (int dx = -r; dx <= r; ++dx) {
                double d2 = (double)dx * dx + (double)dy * dy;
                if (d2 > r2) continue;
                sum += exp(-d2 * inv2s2);
            }
        out[r] = (float)sum;
    }
}

/* src/spatial-filter.ts:217-256 (buildSpatialKernel) for the gaussian
 * shape (support 1.5, evalShape = exp(-2x^2), spatial-filter.ts:63-70).
 * Returns fwidth (3..17) or -1 on bad input. */
OR_EXPORT int or_spatial_kernel_gaussian(double radius, int os, float *out) {
    if (!(radius > 0) || os < 1) return -1;
    const double SUPP = 1.5;
    double fw = 2.0 * SUPP * os * radius;
    int fwidth = (int)floor(fw) + 1;
    if (((fwidth ^ os) & 1) != 0) fwidth++;
    if (fwidth < 3) fwidth = 3;
    if (fwidth > 17) fwidth = 17;
    double adjust = fw > 0 ? (SUPP * fwidth) / fw : 1.0;
    double vals[17], sum = 0.0;
    for (int i = 0; i < fwidth; ++i) {
        double x = ((2.0 * i + 1.0) / fwidth - 1.0) * adjust;
        vals[i] = exp(-2.0 * x * x);
        sum += vals[i];
    }
    /* JS stores each tap into a Float32Array and then divides the f32 value
     * by the double sum, storing f32 again. */
    for (int i = 0; i < fwidth; ++i) {
        float tap = (float)vals[i];
        out[i] = sum != 0 ? (float)((double)tap / sum) : tap;
    }
    return fwidth;
}

/* src/renderer.ts:57-78 (computeDispatch); walkers_override <= 0 = none. */
OR_EXPORT void or_compute_dispatch(double spp, int width, int height, double walkers_override,
                                   double *walkers, double *iters, double *samples) {
    const double TARGET = 1024, MIN_IT = 4096, MAX_IT = 1048576, MAX_W = 65535.0 * 64.0;
    double target = round(spp * width * height);
    /* JS Math.round rounds half up; the products here are integers. */
    double w = walkers_override > 0 ? walkers_override : TARGET;
    double it = ceil(target / w);
    if (walkers_override <= 0) {
        if (it < MIN_IT) {
            it = MIN_IT;
            w = fmax(1.0, ceil(target / it));
        } else if (it > MAX_IT) {
            it = MAX_IT;
            w = fmin(MAX_W, ceil(target / it));
        }
    } else {
        it = fmax(1.0, it);
    }
    *walkers = w; *iters = it; *samples = w * it;
}

/* ----------------------------------------------------------------- splat */
/* Saturating add, chaos.wgsl:8120-8136 (flam3 bump_no_overflow). */
static void or_add_sat(uint32_t *cell, uint32_t delta) {
    if (delta == 0) return;
    uint32_t old = *cell;
    *cell = (0xffffffffu - old) < delta ? 0xffffffffu : old + delta;
}

/* WGSL f32 -> u32 value conversion (clamping, NaN -> 0). */
static uint32_t or_f2u(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967040.0f) return 0xffffffffu;
    return (uint32_t)v;
}

/* Splat of an explicit point stream: chaos.wgsl:8567-8622 + 8699-8718
 * (color_mode 0, no DC override): rotate about (cx, cy), scale, floor,
 * bounds check, palette step/linear lookup, weight = opacity*255, four
 * saturating adds.  pts = n x (x, y, color, opacity). */
OR_EXPORT void or_splat_points(int n, const float *pts, int width, int height, float scale,
                               float cx, float cy, float rotation_rad, int palette_mode,
                               const float *palette, uint32_t *hist) {
    float cos_r = cosf(rotation_rad), sin_r = sinf(rotation_rad);
    for (int k = 0; k < n; ++k) {
        const float *q = pts + (size_t)k * 4;
        float dx = q[0] - cx, dy = q[1] - cy;
        float rx = dx * cos_r - dy * sin_r;
        float ry = dx * sin_r + dy * cos_r;
        float px = rx * scale + (float)width * 0.5f;
        float py = ry * scale + (float)height * 0.5f;
        float fx = floorf(px), fy = floorf(py);
        /* WGSL i32(f) clamps; out-of-range floats fail the bounds test either way. */
        if (!(fx >= 0.0f && fx < (float)width && fy >= 0.0f && fy < (float)height)) continue;
        int xi = (int)fx, yi = (int)fy;
        float c = q[2];
        c = c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c);
        if (q[2] != q[2]) c = 0.0f;
        float cxf = c * 255.0f;
        float pal[4];
        if (palette_mode == 1) {
            uint32_t i0 = or_f2u(cxf);
            float frac = cxf - (float)i0;
            if (i0 >= 255u) { i0 = 254u; frac = 1.0f; }
            for (int ch = 0; ch < 4; ++ch) {
                float a = palette[i0 * 4 + ch], b = palette[(i0 + 1) * 4 + ch];
                pal[ch] = a * (1.0f - frac) + b * frac;
            }
        } else {
            uint32_t idx = or_f2u(cxf);
            if (idx > 255u) idx = 255u;
            for (int ch = 0; ch < 4; ++ch) pal[ch] = palette[idx * 4 + ch];
        }
        float w = q[3] * 255.0f;
        uint32_t *cell = hist + ((size_t)yi * width + xi) * 4;
        or_add_sat(cell + 0, or_f2u(pal[0] * w));
        or_add_sat(cell + 1, or_f2u(pal[1] * w));
        or_add_sat(cell + 2, or_f2u(pal[2] * w));
        or_add_sat(cell + 3, or_f2u(w));
    }
}

/* Pick of an explicit draw stream: chaos.wgsl:8343-8348.  prev < 0 selects
 * the fallback row (stored at row n here). */
OR_EXPORT void or_pick_stream(int n, const uint32_t *rows, int count, const int32_t *prev,
                              const uint32_t *draws, uint32_t *out) {
    for (int k = 0; k < count; ++k) {
        int row = prev[k] >= 0 ? prev[k] : n;
        out[k] = rows[(size_t)row * 16384 + (draws[k] & 16383u)];
    }
}

/* ------------------------------------------------------ density (f32) */
/* density.wgsl:51-123 (density_main), gather form, f32 in WGSL order. */
OR_EXPORT void or_density(int width, int height, float max_rad, float min_rad, float curve,
                          float k1, float k2, const float *knorm, const uint32_t *hist,
                          float *filtered, int row_begin, int row_end) {
    float mr = max_rad < 0 ? 0 : (max_rad > 256.0f ? 256.0f : max_rad);
    int R = (int)ceilf(mr);
    for (int yi = row_begin; yi < row_end; ++yi) {
        for (int xi = 0; xi < width; ++xi) {
            float s0 = 0, s1 = 0, s2 = 0, s3 = 0;
            for (int dy = -R; dy <= R; ++dy) {
                int ny = yi + dy;
                if (ny < 0 || ny >= height) continue;
                for (int dx = -R; dx <= R; ++dx) {
                    int nx = xi + dx;
                    if (nx < 0 || nx >= width) continue;
                    const uint32_t *h = hist + ((size_t)ny * width + nx) * 4;
                    float nc = (float)h[3];
                    if (nc <= 0.0f) continue;
                    float hits = nc / 255.0f;
                    float rf = max_rad / powf(hits + 1.0f, curve);
                    rf = fminf(fmaxf(rf, min_rad), max_rad);
                    int ri = (int)rintf(rf);
                    ri = ri < 0 ? 0 : (ri > 256 ? 256 : ri);
                    float rad = (float)ri;
                    float d2 = (float)(dx * dx + dy * dy);
                    if (d2 > rad * rad) continue;
                    float sig = fmaxf(rad / 3.0f, 1e-6f);
                    float kw = expf(-d2 / (2.0f * sig * sig));
                    float kn = fmaxf(knorm[ri], 1e-6f);
                    float ls = (k1 * logf(1.0f + nc * k2)) / nc;
                    float w = (kw / kn) * ls;
                    s0 = s0 + (float)h[0] * w;
                    s1 = s1 + (float)h[1] * w;
                    s2 = s2 + (float)h[2] * w;
                    s3 = s3 + nc * w;
                }
            }
            float *o = filtered + ((size_t)yi * width + xi) * 4;
            o[0] = s0; o[1] = s1; o[2] = s2; o[3] = s3;
        }
    }
}

/* --------------------------------------------------- visualize (f32) */
typedef struct {
    int width, height, oversample, fwidth;
    float k1, k2, gamma, vibrancy, highpow, linrange;
    float bg[3];
    int transparent;
    unsigned curves_active;   /* composite 1, r 2, g 4, b 8, luma 16 */
    const float *curves;      /* 5 x 256 */
    int hsl_active;
    float hsl_hue, hsl_sat, hsl_light;
} or_viz;

/* visualize_u32.wgsl:51-56 (lut). */
static float or_curve_lut(const float *lut, int ch, float x) {
    float idx = fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f;
    unsigned i0 = (unsigned)floorf(idx);
    unsigned i1 = i0 + 1u < 255u ? i0 + 1u : 255u;
    float t = idx - (float)i0;
    return lut[ch * 256 + i0] * (1.0f - t) + lut[ch * 256 + i1] * t;
}

/* visualize_u32.wgsl:53-72 (rgb2hsv). */
static void or_rgb2hsv(const float c[3], float o[3]) {
    float mx = fmaxf(fmaxf(c[0], c[1]), c[2]);
    float mn = fminf(fminf(c[0], c[1]), c[2]);
    float d = mx - mn, h = 0.0f;
    if (d > 0.0f) {
        if (mx == c[0]) h = (c[1] - c[2]) / d;
        else if (mx == c[1]) h = 2.0f + (c[2] - c[0]) / d;
        else h = 4.0f + (c[0] - c[1]) / d;
        h *= 60.0f;
        if (h < 0.0f) h += 360.0f;
    }
    o[0] = h;
    o[1] = mx > 0.0f ? d / mx : 0.0f;
    o[2] = mx;
}

/* visualize_u32.wgsl:74-90 (hsv2rgb). */
static void or_hsv2rgb(const float c[3], float o[3]) {
    float h = c[0] / 60.0f, s = c[1], v = c[2];
    float i = floorf(h), f = h - i;
    float p = v * (1.0f - s), q = v * (1.0f - s * f), t = v * (1.0f - s * (1.0f - f));
    int ix = (int)i % 6;
    switch (ix) {
        case 0: o[0] = v; o[1] = t; o[2] = p; break;
        case 1: o[0] = q; o[1] = v; o[2] = p; break;
        case 2: o[0] = p; o[1] = v; o[2] = t; break;
        case 3: o[0] = p; o[1] = q; o[2] = v; break;
        case 4: o[0] = t; o[1] = p; o[2] = v; break;
        default: o[0] = v; o[1] = p; o[2] = q; break;
    }
}

/* visualize_u32.wgsl:92-100 (calc_alpha). */
static float or_calc_alpha(float density, float g_inv, float linrange) {
    if (density <= 0.0f) return 0.0f;
    if (density < linrange) {
        float funcval = powf(linrange, g_inv);
        float frac = density / linrange;
        return (1.0f - frac) * density * (funcval / linrange) + frac * powf(density, g_inv);
    }
    return powf(density, g_inv);
}

/* visualize_u32.wgsl:102-128 (calc_newrgb). */
static void or_calc_newrgb(const float c[3], float ls, float highpow, float o[3]) {
    if (ls == 0.0f || (c[0] == 0.0f && c[1] == 0.0f && c[2] == 0.0f)) {
        o[0] = o[1] = o[2] = 0.0f;
        return;
    }
    float sc[3];
    for (int i = 0; i < 3; ++i) sc[i] = ls * (c[i] / 255.0f);
    float maxa = sc[0], maxc = c[0] / 255.0f;
    if (sc[1] > maxa) { maxa = sc[1]; maxc = c[1] / 255.0f; }
    if (sc[2] > maxa) { maxa = sc[2]; maxc = c[2] / 255.0f; }
    if (maxa > 255.0f && highpow >= 0.0f) {
        float newls = 255.0f / maxc;
        float lsratio = powf(newls / ls, highpow);
        float nrgb[3], hsv[3];
        for (int i = 0; i < 3; ++i) nrgb[i] = newls * (c[i] / 255.0f) / 255.0f;
        or_rgb2hsv(nrgb, hsv);
        hsv[1] *= lsratio;
        or_hsv2rgb(hsv, nrgb);
        for (int i = 0; i < 3; ++i) o[i] = nrgb[i] * 255.0f;
    } else {
        float newls = 255.0f / maxc;
        float adjhlp = -highpow;
        if (adjhlp > 1.0f) adjhlp = 1.0f;
        if (maxa <= 255.0f) adjhlp = 1.0f;
        float k = (1.0f - adjhlp) * newls + adjhlp * ls;
        for (int i = 0; i < 3; ++i) o[i] = k * (c[i] / 255.0f);
    }
}

/* visualize_u32.wgsl:147-248 (fs, u32 source, curves/HSL off) and
 * visualize_f32.wgsl:162-271 (fs, DE-filtered f32 source).  src_u32 or
 * src_f32 (exactly one non-NULL) is the super-res RGBA source; out is
 * width x height RGBA f32 in [0,1] (the fragment's return value). */
OR_EXPORT void or_visualize(const or_viz *u, const float *kernel1d, const uint32_t *src_u32,
                            const float *src_f32, float *out, int row_begin, int row_end) {
    int N = u->oversample, fw = u->fwidth, half = fw / 2;
    int sw = u->width * N, sh = u->height * N;
    float g_inv = 1.0f / u->gamma;
    for (int yi = row_begin; yi < row_end; ++yi) {
        for (int xi = 0; xi < u->width; ++xi) {
            float *o = out + ((size_t)yi * u->width + xi) * 4;
            int cx = xi * N + N / 2, cy = yi * N + N / 2;
            float s[4] = {0, 0, 0, 0};
            for (int dy = 0; dy < fw; ++dy) {
                float ky = kernel1d[dy];
                int sy = cy + dy - half;
                sy = sy < 0 ? 0 : (sy > sh - 1 ? sh - 1 : sy);
                for (int dx = 0; dx < fw; ++dx) {
                    float kx = kernel1d[dx];
                    int sx = cx + dx - half;
                    sx = sx < 0 ? 0 : (sx > sw - 1 ? sw - 1 : sx);
                    size_t sb = ((size_t)sy * sw + sx) * 4;
                    if (src_u32) {
                        float cnt = (float)src_u32[sb + 3];
                        if (cnt > 0.0f) {
                            float ls = (u->k1 * logf(1.0f + cnt * u->k2)) / cnt;
                            float w = kx * ky;
                            float v0 = (float)src_u32[sb + 0] * ls, v1 = (float)src_u32[sb + 1] * ls;
                            float v2 = (float)src_u32[sb + 2] * ls, v3 = cnt * ls;
                            s[0] = s[0] + v0 * w; s[1] = s[1] + v1 * w;
                            s[2] = s[2] + v2 * w; s[3] = s[3] + v3 * w;
                        }
                    } else {
                        float w = kx * ky;
                        for (int c = 0; c < 4; ++c) s[c] = s[c] + src_f32[sb + c] * w;
                    }
                }
            }
            if (s[3] <= 0.0f) {
                if (u->transparent) { o[0] = o[1] = o[2] = o[3] = 0.0f; }
                else { o[0] = u->bg[0]; o[1] = u->bg[1]; o[2] = u->bg[2]; o[3] = 1.0f; }
                continue;
            }
            float tmp = s[3] / 255.0f;
            float alpha = or_calc_alpha(tmp, g_inv, u->linrange);
            float ls_alpha = u->vibrancy * 256.0f * alpha / fmaxf(tmp, 1e-12f);
            alpha = fminf(fmaxf(alpha, 0.0f), 1.0f);
            float nrgb[3];
            or_calc_newrgb(s, ls_alpha, u->highpow, nrgb);
            for (int c = 0; c < 3; ++c) {
                float perch = (1.0f - u->vibrancy) * 256.0f * powf(fmaxf(s[c] / 255.0f, 0.0f), g_inv);
                float bg = u->transparent ? 0.0f : (1.0f - alpha) * 256.0f * u->bg[c];
                float comp = nrgb[c] + perch + bg;
                float v = comp / 256.0f;
                o[c] = fminf(fmaxf(v, 0.0f), 1.0f);
            }
            if (u->curves_active && u->curves) {  /* visualize_u32.wgsl:217-231 */
                if (u->curves_active & 16u) {
                    float l = o[0] * 0.299f + o[1] * 0.587f + o[2] * 0.114f;
                    float ln = or_curve_lut(u->curves, 4, l);
                    if (l > 0.0f) { float k = ln / l; o[0] *= k; o[1] *= k; o[2] *= k; }
                }
                if (u->curves_active & 2u) o[0] = or_curve_lut(u->curves, 1, o[0]);
                if (u->curves_active & 4u) o[1] = or_curve_lut(u->curves, 2, o[1]);
                if (u->curves_active & 8u) o[2] = or_curve_lut(u->curves, 3, o[2]);
                if (u->curves_active & 1u)
                    for (int c = 0; c < 3; ++c) o[c] = or_curve_lut(u->curves, 0, o[c]);
            }
            if (u->hsl_active) {  /* visualize_u32.wgsl:234-243 */
                float hsv[3];
                or_rgb2hsv(o, hsv);
                hsv[0] = hsv[0] + u->hsl_hue;
                hsv[0] = hsv[0] - 360.0f * floorf(hsv[0] / 360.0f);
                hsv[1] = fminf(fmaxf(hsv[1] * u->hsl_sat, 0.0f), 1.0f);
                hsv[2] = fminf(fmaxf(hsv[2] + u->hsl_light, 0.0f), 1.0f);
                or_hsv2rgb(hsv, o);
            }
            for (int c = 0; c < 3; ++c) o[c] = fminf(fmaxf(o[c], 0.0f), 1.0f);
            o[3] = u->transparent ? alpha : 1.0f;
        }
    }
}

/* src/export-linear.ts:24-47 (histogramToLinearRgba). */
OR_EXPORT void or_histogram_to_linear(const uint32_t *super_rgba, int width, int height, int os,
                                      double k1, double k2, float *out) {
    int sw = width * os;
    double scale = (k1 * k2) / (double)(os * os);
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            double r = 0, g = 0, b = 0, c = 0;
            for (int sy = 0; sy < os; ++sy)
                for (int sx = 0; sx < os; ++sx) {
                    size_t si = ((size_t)(y * os + sy) * sw + (x * os + sx)) * 4;
                    r += super_rgba[si]; g += super_rgba[si + 1];
                    b += super_rgba[si + 2]; c += super_rgba[si + 3];
                }
            float *o = out + ((size_t)y * width + x) * 4;
            o[0] = (float)(r * scale); o[1] = (float)(g * scale); o[2] = (float)(b * scale);
            o[3] = (float)clamp01d(c * scale);
        }
}
