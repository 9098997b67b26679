/*
 * pyr3-b200 C-ABI: the drop-in boundary that replaces the reference's
 * WebGPU passes under its Renderer API (MattAltermatt/pyr3
 * src/renderer.ts:163-318).  Plain pointers and sizes only; every function
 * returns 0 on success or a negative PYR3_E* code, with a message available
 * from pyr3_last_error().
 *
 * Threading: one renderer handle per host thread.  Work is enqueued on the
 * renderer's CUDA stream and is asynchronous until pyr3_sync() or a call
 * that returns host data (pyr3_read_histogram, pyr3_present to a host
 * buffer, pyr3_counters).
 *
 * Buffers: the caller owns every host buffer it passes; the renderer owns
 * all device memory it allocates (recreated on pyr3_resize).  Entries that
 * take DEVICE pointers say so.
 */
#ifndef PYR3_H
#define PYR3_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PYR3_OK 0
#define PYR3_E_INVALID (-1)   /* bad argument / malformed genome */
#define PYR3_E_CUDA (-2)      /* CUDA runtime or driver error */
#define PYR3_E_NVRTC (-3)     /* JIT compile of the chaos kernel failed */
#define PYR3_E_NOMEM (-4)     /* device allocation failed */
#define PYR3_E_UNSUPPORTED (-5) /* variation index not implemented by this library */

#define PYR3_XFORM_FLOATS 116  /* packed xform record (src/genome.ts:293-313) */
#define PYR3_MAX_XFORMS 128    /* src/genome.ts:326 */
#define PYR3_PALETTE_FLOATS 1024 /* 256 x RGBA f32 (src/palette.ts:211) */

typedef struct pyr3_renderer pyr3_renderer;

/* createRenderer options (src/renderer.ts:78-86). */
typedef struct {
  uint32_t width, height; /* output canvas */
  uint32_t oversample;    /* >= 1; super-res canvas = width*os x height*os */
  float filter_radius;    /* spatial filter radius in output px; <= 0 -> 0.5 */
  int32_t device;         /* CUDA device ordinal */
} pyr3_opts;

/* A genome as the reference's chaos pass receives it after
 * expandGenomeForGPU (src/symmetry.ts:21) and packXforms
 * (src/genome.ts:408): n_xforms regular records followed, when
 * final_slot >= 0, by the final xform record at slot n_xforms. */
typedef struct {
  const float *xforms;    /* (n_xforms + (final_slot >= 0)) x 116 f32 */
  uint32_t n_xforms;      /* 1..128 */
  int32_t final_slot;     /* -1 or n_xforms (src/genome.ts:432) */
  const float *xaos;      /* n_xforms x n_xforms row-major or NULL */
  float scale, cx, cy;    /* viewport (pixels per unit at output res) */
  float rotate_deg;       /* CCW camera rotation */
  uint32_t palette_mode;  /* 0 step (flam3 default), 1 linear */
  float xform_blend;      /* 0..1 (chaos.wgsl:8372) */
} pyr3_genome;

/* iterate() request (src/renderer.ts:127-146 + chaos.ts:381-456). */
typedef struct {
  uint64_t walkers;        /* reference walker count for this chunk */
  uint64_t iters_per_walker;
  uint32_t seed;
  float walker_jitter;     /* < 0 -> default 1e-7 */
  uint32_t color_mode;     /* 0 palette, 1 flow, 2 trap, 3 phase */
  float flow_strength, flow_scale;
  uint32_t trap_kind, trap_mode;
  float trap_cx, trap_cy, trap_radius, trap_angle_deg, trap_falloff, trap_freq, trap_strength;
  float phase_strength, phase_freq;
  uint32_t flags;          /* PYR3_ITER_* */
} pyr3_iterate_opts;

/* Use exactly `walkers` ISAAC streams x `iters_per_walker` iterations, as
 * the reference dispatch does.  Without it the renderer keeps the sample
 * total walkers*iters but spreads it over its own persistent walker pool
 * (each stream still seeded by the reference's packIsaacStates rule). */
#define PYR3_ITER_EXACT_WALKERS 1u
/* Pool every distinct histogram bucket of a warp (__match_any_sync) instead
   of only the warp's hot bucket. */
#define PYR3_ITER_AGGREGATE 2u
/* Chaos kernel.  Without a kernel flag an autotuner picks, per genome
 * structure, the fastest on the first launch of at least 2^26 samples (that
 * launch then waits for its trial runs), and smaller launches before that
 * use the barrier kernel.  The barrier kernel runs each round of a CTA's
 * walkers in xform order between barriers; the queue kernel (genomes of up
 * to 32 xforms) keeps per-xform walker queues so warps run one xform at a
 * time without barriers; the wave kernel (genomes of up to 32 xforms) keeps
 * every walker of the launch in device memory grouped by next xform and
 * advances all of them one iteration per launch.  A kernel that cannot
 * serve a genome or a request falls back to the barrier kernel. */
#define PYR3_ITER_KERNEL_BARRIER 4u
#define PYR3_ITER_KERNEL_QUEUE 8u
#define PYR3_ITER_KERNEL_WAVE 16u

/* present() request (src/renderer.ts:148-158, visualize.ts:178-204). */
typedef struct {
  float gamma, vibrancy, highpow, brightness, linrange; /* src/tonemap.ts */
  int32_t density_on;       /* 1 -> density estimation pass */
  float de_max_rad, de_min_rad, de_curve;               /* src/density.ts */
  float background[3];
  int32_t transparent;
  double scale;             /* genome.scale (calibration k2) */
  /* Colour curves (src/channel-curves.ts, visualize_u32.wgsl:217-231):
   * bit mask composite 1, r 2, g 4, b 8, luma 16 (0 = off) and the baked
   * 5 x 256 f32 LUT in host memory (read only when the mask is non-zero). */
  uint32_t curves_active;
  const float *curves;
  /* HSL adjustment (visualize_u32.wgsl:234-243; src/visualize.ts:194-198):
   * hue offset in degrees, saturation multiplier and lightness addend
   * (the genome's percentages / 100). */
  int32_t hsl_active;
  float hsl_hue, hsl_sat, hsl_light;
} pyr3_present_opts;

#define PYR3_OUT_RGBA8 0      /* W x H x 4 u8 (rgba8unorm) */
#define PYR3_OUT_RGBA32F 1    /* W x H x 4 f32 (fragment value) */
#define PYR3_OUT_RGBA16F 2    /* W x H x 4 binary16, nearest even (the rgba16float
                                 texture of the png16 and exr exports) */
#define PYR3_OUT_PNG16 3      /* W x H x 4 u16: displayHalfToPng16
                                 (src/gpu-readback.ts:106-115) of the rgba16float value */
#define PYR3_OUT_EXR_DISPLAY 4 /* W x H x 4 f32: displayHalfToLinearExr
                                 (src/gpu-readback.ts:83-104): sRGB-to-linear RGB of
                                 the clamped rgba16float value, alpha clamped */

typedef struct pyr3_batch pyr3_batch;

/* ---- lifecycle -------------------------------------------------------- */
/* createRenderer (src/renderer.ts:214). */
int pyr3_create(const pyr3_opts *opts, pyr3_renderer **out);
/* Renderer.destroy (src/renderer.ts:316). */
int pyr3_destroy(pyr3_renderer *r);
/* Renderer.resize (src/renderer.ts:281). */
int pyr3_resize(pyr3_renderer *r, const pyr3_opts *opts);
/* Last error message of the calling thread ("" if none). */
const char *pyr3_last_error(void);

/* ---- the render path -------------------------------------------------- */
/* Renderer.reset (src/renderer.ts:221): upload the palette (256 x RGBA f32,
 * the bakeLUT output of src/palette.ts:71) and zero the histogram. */
int pyr3_reset(pyr3_renderer *r, const float *palette);
/* Renderer.iterate (src/renderer.ts:227) -> chaos.dispatch
 * (src/chaos.ts:333): accumulate walkers*iters post-fuse samples. */
int pyr3_iterate(pyr3_renderer *r, const pyr3_genome *g, const pyr3_iterate_opts *o);
/* Renderer.present (src/renderer.ts:241): density estimation (optional) +
 * tonemap of the accumulated histogram.  total_samples = sum of
 * walkers*iters since reset.  `out` is a HOST buffer of W*H pixels of
 * out_kind (PYR3_OUT_*: 4, 16, 8, 8 or 16 bytes each); the call returns
 * after the copy.  The png16 and exr kinds are written by the tonemap pass
 * itself, in place of the reference's host-side transforms of its
 * rgba16float readback. */
int pyr3_present(pyr3_renderer *r, const pyr3_present_opts *p, uint64_t total_samples,
                 void *out, int32_t out_kind);
/* Same as pyr3_present but writes into a DEVICE buffer and returns without
 * synchronising. */
int pyr3_present_device(pyr3_renderer *r, const pyr3_present_opts *p, uint64_t total_samples,
                        void *device_out, int32_t out_kind);
/* Renderer.readHistogram (src/renderer.ts:209, src/chaos.ts:293): raw
 * super-res histogram, superW*superH*4 u32 (R, G, B, count). */
int pyr3_read_histogram(pyr3_renderer *r, uint32_t *host_out);
/* histogramToLinearRgba (src/export-linear.ts:24-47) of the current
 * histogram, computed on the device: width x height x RGBA f32 linear,
 * scene-referred values (k1, k2 from deriveCalibration, src/calibration.ts). */
int pyr3_read_linear(pyr3_renderer *r, double k1, double k2, float *host_out);
/* An rgba32f fragment-value image already on the device (e.g. from
 * pyr3_present_device) written as another output kind, with the same
 * per-pixel steps as the tonemap's store: one present can feed several
 * exports.  Both buffers 16-byte aligned; runs on `stream` (a cudaStream_t,
 * NULL = default stream) of the current device. */
int pyr3_convert_display(const void *device_rgba32f, uint64_t pixels, int32_t out_kind,
                         void *device_out, void *stream);

/* ---- auto-exposure ----------------------------------------------------- */
/* Constants of src/auto-exposure.ts:43-61: the probe's long edge, quality
 * and seed, the no-op deadband, the refinement cap and the brightness
 * clamp. */
#define PYR3_AE_PROBE_LONG_EDGE 1024
#define PYR3_AE_PROBE_QUALITY 16
#define PYR3_AE_PROBE_SEED 0x9e3779b9u
#define PYR3_AE_DEADBAND 0.10
#define PYR3_AE_MAX_ITERS 4
#define PYR3_AE_BRIGHTNESS_MIN 1e-3
#define PYR3_AE_BRIGHTNESS_MAX 1e4

/* BrightnessFit (src/auto-exposure.ts:131-142). */
typedef struct {
  double brightness;  /* brightness to present the final image at */
  int32_t corrected;  /* 1 iff brightness differs from the base */
  int32_t iters;      /* re-presents performed */
  double final_mean;  /* last measured mean luminance */
  double factor;      /* target / initial mean (diagnostic) */
} pyr3_brightness_fit;

/* rerender(b, &mean, ctx): present at brightness b, store the measured mean
 * luminance and return 0, or return a non-zero error code (which ends the
 * fit and is returned). */
typedef int (*pyr3_rerender_fn)(double brightness, double *mean, void *ctx);

/* fitBrightnessToTarget (src/auto-exposure.ts:147-175), host logic only:
 * fixed-point fit of the brightness so the measured mean luminance reaches
 * target_mean, starting from initial_mean measured at base_brightness.
 * No-op (fit->corrected = 0, no rerender call) inside the deadband or for a
 * non-finite or non-positive target / initial mean. */
int pyr3_fit_brightness(double base_brightness, double target_mean, double initial_mean,
                        pyr3_rerender_fn rerender, void *ctx, pyr3_brightness_fit *fit);
/* computeMeanLuminance / computeMeanLuminanceHalf (src/auto-exposure.ts:
 * 70-97) of a DEVICE image of `pixels` RGBA pixels, on the renderer's
 * stream; returns after the result is read back.  kind PYR3_OUT_RGBA8: mean
 * of (R+G+B)/3 in [0, 255].  kind PYR3_OUT_RGBA16F: computeMeanLuminanceHalf
 * (non-finite -> 0, clamped to [0, 1], x 255).  kind PYR3_OUT_RGBA32F: the
 * same after rounding each channel to binary16 (the rgba16float texture
 * the reference reads back).  0 pixels -> 0.  The image must be 16-byte
 * aligned.  The sum is exact (integers on the device), so the mean
 * is the same on every run. */
int pyr3_mean_luminance(pyr3_renderer *r, const void *device_img, uint64_t pixels, int32_t kind,
                        double *mean);
/* The auto-exposure re-present loop of bin/pyr3-render.ts:487-513 on the
 * device: present at p->brightness into device_out (W x H, out_kind
 * PYR3_OUT_RGBA8, PYR3_OUT_RGBA16F or PYR3_OUT_RGBA32F),
 * measure its mean luminance, then fitBrightnessToTarget with every
 * re-present and measurement on the device (only the 8-byte luminance sum
 * is read back per pass).  On return device_out holds the image at
 * fit->brightness; k1 is derived from that brightness in double, as the
 * reference's genome holds it.  target_mean comes from a probe render
 * (measureProbeLuminance, src/auto-exposure.ts:99-129: the genome at
 * PYR3_AE_PROBE_LONG_EDGE, PYR3_AE_PROBE_QUALITY spp, oversample 1, seed
 * PYR3_AE_PROBE_SEED, measured with pyr3_mean_luminance). */
int pyr3_auto_exposure(pyr3_renderer *r, const pyr3_present_opts *p, uint64_t total_samples,
                       double target_mean, void *device_out, int32_t out_kind,
                       pyr3_brightness_fit *fit);

/* ---- batches ---------------------------------------------------------- */
/* Batched rendering of many genomes (no counterpart in the reference,
 * which renders genomes one dispatch at a time): genomes too small to fill
 * the GPU share one CUDA graph, genomes of 2^24 samples or more run beside
 * it through pyr3_iterate, one after another.  renderers[i] renders
 * genomes[i] with opts[i] (walkers x iters_per_walker samples; without
 * PYR3_ITER_EXACT_WALKERS the batch picks its own walker count per genome).
 * All renderers must be on one device.  pyr3_batch_run clears every
 * renderer's histogram and accumulates its samples, asynchronously, on the
 * batch's own stream; after pyr3_batch_sync each renderer can be presented
 * or read.  Genome values are captured at creation. */
int pyr3_batch_create(pyr3_renderer *const *renderers, const pyr3_genome *genomes,
                      const pyr3_iterate_opts *opts, uint32_t n, uint32_t n_streams,
                      pyr3_batch **out);
int pyr3_batch_run(pyr3_batch *b);
/* Wait for the last run; its device time (ms) and total samples. */
int pyr3_batch_sync(pyr3_batch *b, float *ms, uint64_t *samples);
int pyr3_batch_destroy(pyr3_batch *b);

/* Renderer.readIndexMap (src/renderer.ts:205): superW*superH u32 colour
 * index sums (valid after iterating with capture on). */
int pyr3_read_index_map(pyr3_renderer *r, uint32_t *host_out);
/* Renderer.setCaptureIndex (src/renderer.ts:200). */
int pyr3_set_capture_index(pyr3_renderer *r, int32_t on);
/* Wait for all work queued on the renderer. */
int pyr3_sync(pyr3_renderer *r);
/* Super-res dimensions and device histogram pointer (for callers that keep
 * data on the GPU). */
int pyr3_info(pyr3_renderer *r, uint32_t *super_w, uint32_t *super_h, void **device_hist);
/* Accepted post-fuse samples and in-canvas splats since reset. */
int pyr3_counters(pyr3_renderer *r, uint64_t *samples, uint64_t *splats);
/* Device time in ms of the last pyr3_iterate chaos launch (CUDA events). */
int pyr3_last_iterate_ms(pyr3_renderer *r, float *ms);
/* Kernel launches the last pyr3_iterate issued (the wave kernel issues one
 * per iteration; autotuner trials included). */
int pyr3_last_iterate_launches(pyr3_renderer *r, uint64_t *launches);

/* CUDA-event timing on the renderer's stream: record mark `slot` (0..7),
 * then read the device time between two marks (waits for the later one). */
int pyr3_mark(pyr3_renderer *r, int32_t slot);
int pyr3_elapsed(pyr3_renderer *r, int32_t a, int32_t b, float *ms);
/* Measurement: device time (*ms) of `splats` deposits of 4 saturating u32
 * atomics, the chaos kernel's scatter, into uniformly random cells of the
 * renderer's histogram -- the random-scatter rate its splats are measured
 * against.  Leaves the histogram's contents changed (call pyr3_reset). */
int pyr3_splat_rate(pyr3_renderer *r, uint64_t splats, float *ms);
/* Overwrite a scratch buffer of `bytes` on the renderer's stream (evicts
 * the L2 between timed steps). */
int pyr3_flush_l2(pyr3_renderer *r, uint64_t bytes);

/* ---- stage entry points (parity tests and tools) ---------------------- */
/* packIsaacStates (src/isaac.ts:194) computed on the device: n x 36 u32 in
 * the reference layout for walkers base..base+n-1. */
int pyr3_seed_walkers(uint32_t seed, uint64_t base, uint32_t n, uint32_t *host_out);
/* Evaluate one variation (apply_variation, chaos.wgsl:7731) on n points on
 * the device; isaac (n x 36 u32, reference layout) is each point's RNG
 * stream and is updated in place. params10/a0/a1 as in the packed xform. */
int pyr3_eval_variation(uint32_t idx, uint32_t n, const float *pts_xy, float weight,
                        const float *params10, const float *a0, const float *a1,
                        uint32_t *isaac, float *out_xy);
/* Direct colour of a DC variation (dc_color_for, chaos.wgsl:8192) at n
 * points; hit[i] = 1 when the variation colours the point. */
int pyr3_eval_dc_color(uint32_t idx, uint32_t n, const float *pts_xy, const float *v4,
                       const float *ve4, float *out_rgb, int32_t *hit);
/* Xform pick of an explicit draw stream (chaos.wgsl:8343): prev[i] < 0
 * selects the no-prior row.  weights / xaos as in pyr3_genome. */
int pyr3_pick_stream(uint32_t n_xforms, const float *weights, const float *xaos,
                     uint32_t count, const int32_t *prev, const uint32_t *draws,
                     uint32_t *out);
/* Splat an explicit point stream (x, y, colour, opacity per point) into a
 * zeroed width x height x 4 u32 histogram with the chaos kernel's
 * saturating scatter (chaos.wgsl:8567-8718, colour mode 0). */
int pyr3_splat_points(uint32_t n, const float *pts, uint32_t width, uint32_t height,
                      float scale, float cx, float cy, float rotation_rad,
                      uint32_t palette_mode, const float *palette, int32_t aggregate,
                      uint32_t *hist_inout);
/* Density estimation + tonemap of a given super-res histogram (no chaos
 * pass): out = width x height x RGBA f32. */
int pyr3_density_tonemap(const uint32_t *hist, uint32_t width, uint32_t height,
                         uint32_t oversample, float filter_radius, const pyr3_present_opts *p,
                         uint64_t total_samples, float *out_rgba, float *filtered_out);
/* Allocation-free density estimation + tonemap.  No counterpart in the
 * reference: it is for callers that cannot allocate device memory -- code
 * inside another engine's frame loop or memory pool, or code that must not
 * allocate once running.  The caller passes a super-res histogram already
 * on the device (superW x superH x 4 u32) and a device output image
 * (width x height, any PYR3_OUT_* kind); the intermediate
 * density output and lookup tables live in one fixed array inside the
 * library (about 16.4 MiB, held by every GPU that loads the library until
 * the process exits).  Limit: width*height*oversample^2 <= 1,048,576
 * super-sampled pixels, larger canvases fail with PYR3_E_INVALID.  Runs on
 * `stream` (a cudaStream_t, NULL = default stream) of the current device.
 * The first call on a device sets the array up, on `stream`, and waits for
 * that set-up to finish, so make the first call before any stream capture
 * begins.  Each call hands its filter taps and curves LUT to the device as
 * a kernel parameter, so `p` and its curves need not outlive the call.
 * All calls share the array: calls whose GPU work overlaps race and must
 * be serialised by the caller. */
int pyr3_density_tonemap_noalloc(const uint32_t *device_hist, uint32_t width, uint32_t height,
                                 uint32_t oversample, float filter_radius,
                                 const pyr3_present_opts *p, uint64_t total_samples,
                                 void *device_out, int32_t out_kind, void *stream);
/* Compile (or fetch from cache) the chaos kernel for a genome structure;
 * returns the NVRTC log on failure via pyr3_last_error. */
int pyr3_prepare(pyr3_renderer *r, const pyr3_genome *g);

/* ---- learned denoiser layers ---------------------------------------- */
/* No counterpart in the reference: the denoiser is an addition.  Layers of
 * a U-Net over device tensors, NCHW f32; each operand is a device pointer
 * plus its per-image stride in floats, so a channel slice of a larger
 * tensor (a skip concatenation) is a valid operand.  Work is queued on
 * `stream` (a cudaStream_t, NULL = legacy default stream).  Errors:
 * PYR3_E_INVALID for null operands or bad sizes, PYR3_E_CUDA for launch
 * failures. */
/* out[n,co] = bias[co] + sum_ci conv3x3(in[n,ci], weight[co][ci]), zero
 * padding; ReLU if relu.  weight is [co][ci][3][3]; bias may be NULL. */
int pyr3_dn_conv3x3(const float *in, int64_t in_ns, int32_t ci, float *out, int64_t out_ns,
                    int32_t co, int32_t n, int32_t h, int32_t w, const float *weight,
                    const float *bias, int32_t relu, void *stream);
/* pyr3_dn_conv3x3 on the tensor cores (tcgen05): input and weights rounded
 * to bf16, products accumulated in f32; co <= 128 (PYR3_E_INVALID above). */
int pyr3_dn_conv3x3_bf16(const float *in, int64_t in_ns, int32_t ci, float *out, int64_t out_ns,
                         int32_t co, int32_t n, int32_t h, int32_t w, const float *weight,
                         const float *bias, int32_t relu, void *stream);
/* Weight (and, if dbias is not NULL, bias) gradient of pyr3_dn_conv3x3
 * given its input and the gradient of its output; overwrites.  The sum
 * over pixels is split into partials held in `scratch`, a device buffer
 * of at least pyr3_dn_wgrad_scratch_floats(co, ci) floats (PYR3_E_INVALID
 * if smaller), and added in a fixed order, so the result is reproducible. */
int pyr3_dn_conv3x3_wgrad(const float *in, int64_t in_ns, int32_t ci, const float *dout,
                          int64_t dout_ns, int32_t co, int32_t n, int32_t h, int32_t w,
                          float *dweight, float *dbias, float *scratch, uint64_t scratch_floats,
                          void *stream);
/* pyr3_dn_conv3x3_wgrad on the tensor cores (tcgen05): per tap a GEMM over
 * pixel positions with input and output gradient rounded to bf16 and f32
 * accumulation; co, ci <= 128 and n <= 128 (PYR3_E_INVALID otherwise), the
 * same scratch. */
int pyr3_dn_conv3x3_wgrad_bf16(const float *in, int64_t in_ns, int32_t ci, const float *dout,
                               int64_t dout_ns, int32_t co, int32_t n, int32_t h, int32_t w,
                               float *dweight, float *dbias, float *scratch, uint64_t scratch_floats,
                               void *stream);
/* Floats of scratch pyr3_dn_conv3x3_wgrad(_bf16) needs for co x ci channels
 * (0 for non-positive sizes). */
uint64_t pyr3_dn_wgrad_scratch_floats(int32_t co, int32_t ci);
/* flipped[ci][co][k] = weight[co][ci][8-k]: pyr3_dn_conv3x3 with these
 * weights (co and ci swapped, no bias) maps an output gradient to the
 * input gradient. */
int pyr3_dn_flip_weights(const float *weight, int32_t co, int32_t ci, float *flipped, void *stream);
/* grad = 0 wherever y <= 0 (ReLU backward), c channels of hw pixels. */
int pyr3_dn_relu_mask(float *grad, int64_t grad_ns, const float *y, int64_t y_ns, int32_t c,
                      int32_t n, int32_t hw, void *stream);
/* y += x over c channels of hw pixels. */
int pyr3_dn_add(float *y, int64_t y_ns, const float *x, int64_t x_ns, int32_t c, int32_t n,
                int32_t hw, void *stream);
/* 2x2 average pool of an h x w input (h, w even); with backward, in is the
 * (h/2 x w/2) output gradient and out the h x w input gradient, written or,
 * with accumulate, added. */
int pyr3_dn_pool2(const float *in, int64_t in_ns, float *out, int64_t out_ns, int32_t c, int32_t n,
                  int32_t h, int32_t w, int32_t backward, int32_t accumulate, void *stream);
/* Nearest 2x upsample of an h x w input; with backward, in is the
 * (2h x 2w) output gradient and out the h x w input gradient. */
int pyr3_dn_up2(const float *in, int64_t in_ns, float *out, int64_t out_ns, int32_t c, int32_t n,
                int32_t h, int32_t w, int32_t backward, void *stream);
/* grad = 2 (pred - target) / count; *loss_sum += sum (pred - target)^2
 * (device float, zeroed by the caller). */
int pyr3_dn_mse(const float *pred, const float *target, int64_t count, float *grad,
                float *loss_sum, void *stream);
/* One bias-corrected Adam step (step >= 1) over count parameters. */
int pyr3_dn_adam(float *param, const float *grad, float *m, float *v, int64_t count, float lr,
                 float beta1, float beta2, float eps, int32_t step, void *stream);

/* ---- build checks (no GPU needed) ------------------------------------ */
/* Generate + NVRTC-compile the chaos kernel for a genome structure without
 * touching a device; *cubin_bytes receives the image size. */
int pyr3_jit_compile(const pyr3_genome *g, int32_t aggregate, uint64_t *cubin_bytes);
/* Copy the generated NVRTC source for a genome into buf (size cap); returns
 * the full length through *len. */
int pyr3_jit_source(const pyr3_genome *g, char *buf, uint64_t cap, uint64_t *len);
/* NVRTC-compile the variation evaluator for `idx` (no device). */
int pyr3_jit_compile_variation(uint32_t idx, uint64_t *cubin_bytes);
/* The (n+1) x 16384 xform pick table (src/genome.ts:482-534; row n = the
 * no-prior row) as the renderer reproduces it from its per-row boundaries. */
int pyr3_pick_table(uint32_t n_xforms, const float *weights, const float *xaos,
                    uint32_t *table_out);
/* 1 if this library implements variation idx, 0 if not; name via *name. */
int pyr3_variation_info(uint32_t idx, int32_t *implemented, int32_t *is_dc, const char **name);

#ifdef __cplusplus
}
#endif
#endif /* PYR3_H */
