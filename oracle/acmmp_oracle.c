/* The live path's PatchMatch estimator (ACMMP-style) restated in C: one
 * pyramid level per call, with the upsampling from the coarser level and
 * the geometric consistency against previous-level depths (the level loop
 * and the cluster's links are driven from oracle/__init__.py); no SfM
 * planar prior.  TEST INFRASTRUCTURE ONLY.
 *
 * Follows opensfm/src/lib/dense/src/estimator.cc:120-243 (Run / RunLevel:
 * random initialisation, then per iteration a red and a black PatchMatch
 * pass and a red and a black checkerboard filter), 473-558 (the launches),
 * 941-1040 (ReadBackResults: depth and normal from the planes, 5x5 median
 * rejection, logistic confidence) and the kernels of opencl_kernels.h:
 * 44-137 (RNG, camera helpers), 157-237 (strided bilateral NCC), 491-574
 * (multi-scale NCC, census), 585-750 (single-source and per-view costs),
 * 752-829 (initial cost and top-k views), 831-1053 (CDF, smoothness,
 * weighted cost), 1055-1124 (random init), 1298-1826 (PatchMatch pass) and
 * 1897-2099 (checkerboard filter).
 *
 * The reference runs these as OpenCL kernels, unavailable here, whose
 * float results depend on the device (hardware-filtered image reads,
 * exp/log/normalize precision, contraction).  Parity is unpinned by the
 * reference's outputs; this file fixes one arithmetic instead, which the
 * library's kernels match bit for bit:
 *   - FP32, every operation rounded by itself in the written order (no
 *     contraction), except the fmaf written out in the NCC tap, the
 *     bilinear blend and acm_exp (rounded once, as the kernels' fused
 *     multiply-adds); IEEE division and square root;
 *   - exp and log by the functions below (Cody-Waite reduction and fixed
 *     polynomials), not the C library's;
 *   - images as float(v) * float(1/255) (cv::Mat::convertTo with 1/255);
 *   - read_imagef with a linear filter and clamp-to-edge as the OpenCL
 *     specification writes it, with exact fractions (hardware filters
 *     quantise them) and coordinates beyond 16 texels outside the image
 *     (or NaN) moved to 16 texels outside;
 *   - normalize(v) = v / sqrt((x*x + y*y) + z*z), v itself when the
 *     length is 0.
 * The confidence of the readback uses the C library's expf, as the
 * reference's host code does.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ACM_MAX_SRC 16

/* ------------------------------------------------------------ arithmetic */
static float acm_ldexp(float p, int n) {
  /* p * 2^n for p in [0.5, 2], n in [-151, 128], two exact steps. */
  int n1 = n / 2, n2 = n - n1;
  union {
    uint32_t u;
    float f;
  } a, b;
  if (n1 < -126 || n2 < -126 || n1 > 127 || n2 > 127) {
    if (n < 0) return 0.0f;
    return INFINITY;
  }
  a.u = (uint32_t)(n1 + 127) << 23;
  b.u = (uint32_t)(n2 + 127) << 23;
  return (p * a.f) * b.f;
}

/* e^x: n = round(x log2 e), r = x - n ln2 (two-part ln2), e^r by its
 * degree-7 Taylor polynomial in Horner form (|r| <= 0.347); the reduction
 * and the Horner steps are fused multiply-adds (fmaf, rounded once). */
float acm_exp(float x) {
  if (x != x) return x;
  if (x > 88.72283f) return INFINITY;
  if (x < -103.97208f) return 0.0f;
  const float t = x * 1.44269502f;
  const float nf = floorf(t + 0.5f);
  const int n = (int)nf;
  const float r = fmaf(-nf, 1.42860677e-06f, fmaf(-nf, 0.693145752f, x));
  float p = 1.98412701e-04f;
  p = fmaf(p, r, 1.38888892e-03f);
  p = fmaf(p, r, 8.33333377e-03f);
  p = fmaf(p, r, 4.16666679e-02f);
  p = fmaf(p, r, 1.66666672e-01f);
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  return acm_ldexp(p, n);
}

/* ln x for x > 0: x = m 2^e with m in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1),
 * ln m = 2 (s + s^3/3 + ... + s^11/11), ln x = e ln2 + ln m. */
float acm_log(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  union {
    uint32_t u;
    float f;
  } v;
  v.f = x;
  int e = 0;
  if (v.u < 0x00800000u) { /* subnormal: scale by 2^24 */
    v.f = x * 16777216.0f;
    e = -24;
  }
  e += (int)(v.u >> 23) - 127;
  v.u = (v.u & 0x007FFFFFu) | 0x3F800000u; /* m in [1, 2) */
  float m = v.f;
  if (m > 1.41421354f) {
    m = m * 0.5f;
    e += 1;
  }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  float q = 0.0909090936f;
  q = q * s2 + 0.111111112f;
  q = q * s2 + 0.142857149f;
  q = q * s2 + 0.200000003f;
  q = q * s2 + 0.333333343f;
  q = q * s2 + 1.0f;
  const float lnm = 2.0f * (s * q);
  const float ef = (float)e;
  return (ef * 0.693145752f + lnm) + ef * 1.42860677e-06f;
}

static void acm_normalize(float* v) {
  const float len = sqrtf((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
  if (len == 0.0f) return;
  v[0] = v[0] / len;
  v[1] = v[1] / len;
  v[2] = v[2] / len;
}

static float acm_clampf(float x, float lo, float hi) {
  const float m = x > lo ? x : lo; /* fmax / fmin for non-NaN x */
  return m < hi ? m : hi;
}

/* ---------------------------------------------------------------- images */
typedef struct {
  const float* px; /* [H][W], values float(v) * float(1/255) */
  int W, H;
} acm_img;

static int acm_clampi(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

/* read_imagef(img, linear | clamp-to-edge, (u, v)) at unnormalised (u, v). */
static float acm_sample(const acm_img* im, float u, float v) {
  float xm = u - 0.5f, ym = v - 0.5f;
  if (!(xm >= -16.0f)) xm = -16.0f;
  if (!(xm <= (float)im->W + 16.0f)) xm = (float)im->W + 16.0f;
  if (!(ym >= -16.0f)) ym = -16.0f;
  if (!(ym <= (float)im->H + 16.0f)) ym = (float)im->H + 16.0f;
  const float fx = floorf(xm), fy = floorf(ym);
  const float a = xm - fx, b = ym - fy;
  const int i0 = (int)fx, j0 = (int)fy;
  const int xa = acm_clampi(i0, im->W), xb = acm_clampi(i0 + 1, im->W);
  const int ya = acm_clampi(j0, im->H), yb = acm_clampi(j0 + 1, im->H);
  const float t00 = im->px[(size_t)ya * im->W + xa], t10 = im->px[(size_t)ya * im->W + xb];
  const float t01 = im->px[(size_t)yb * im->W + xa], t11 = im->px[(size_t)yb * im->W + xb];
  /* ((w00 t00 + w10 t10) + w01 t01) + w11 t11, the last three fused. */
  const float ia = 1.0f - a, ib = 1.0f - b;
  return fmaf(a * b, t11, fmaf(ia * b, t01, fmaf(a * ib, t10, (ia * ib) * t00)));
}

/* --------------------------------------------------------------- cameras */
typedef struct {
  float K[9], R[9], t[3];
} acm_cam;

static void acm_project(const acm_cam* c, const float* X, float* p) {
  const float xc0 = ((c->R[0] * X[0] + c->R[1] * X[1]) + c->R[2] * X[2]) + c->t[0];
  const float xc1 = ((c->R[3] * X[0] + c->R[4] * X[1]) + c->R[5] * X[2]) + c->t[1];
  const float xc2 = ((c->R[6] * X[0] + c->R[7] * X[1]) + c->R[8] * X[2]) + c->t[2];
  p[0] = (c->K[0] * xc0 + c->K[1] * xc1) + c->K[2] * xc2;
  p[1] = (c->K[3] * xc0 + c->K[4] * xc1) + c->K[5] * xc2;
  p[2] = (c->K[6] * xc0 + c->K[7] * xc1) + c->K[8] * xc2;
}

static void acm_backproject(const acm_cam* c, float x, float y, float depth, float* w) {
  const float px = depth * (x - c->K[2]) / c->K[0];
  const float py = depth * (y - c->K[5]) / c->K[4];
  const float d0 = px - c->t[0], d1 = py - c->t[1], d2 = depth - c->t[2];
  w[0] = (c->R[0] * d0 + c->R[3] * d1) + c->R[6] * d2;
  w[1] = (c->R[1] * d0 + c->R[4] * d1) + c->R[7] * d2;
  w[2] = (c->R[2] * d0 + c->R[5] * d1) + c->R[8] * d2;
}

static float acm_depth_from_plane(const acm_cam* c, float x, float y, const float* pl) {
  const float denom = (pl[0] * (x - c->K[2]) / c->K[0] + pl[1] * (y - c->K[5]) / c->K[4]) + pl[2];
  if (fabsf(denom) < 1e-6f) return 0.0f;
  return -pl[3] / denom;
}

static void acm_plane_from_depth_normal(const acm_cam* c, float x, float y, float depth,
                                        const float* n, float* pl) {
  const float p0 = depth * (x - c->K[2]) / c->K[0];
  const float p1 = depth * (y - c->K[5]) / c->K[4];
  const float p2 = depth;
  pl[0] = n[0];
  pl[1] = n[1];
  pl[2] = n[2];
  pl[3] = -((n[0] * p0 + n[1] * p1) + n[2] * p2);
}

/* Philox-style generator (opencl_kernels.h:47-66): four rounds. */
static float acm_rand(uint32_t* st, uint32_t key) {
  for (uint32_t i = 0; i < 4; ++i) {
    const uint32_t k = key + i * 0x9E3779B9u;
    const uint64_t prod = (uint64_t)st[0] * 0xD256D193u;
    const uint32_t lo = (uint32_t)prod, hi = (uint32_t)(prod >> 32);
    const uint32_t nx = st[1] ^ k ^ hi;
    st[0] = nx;
    st[1] = lo;
  }
  return (float)st[0] / 4294967296.0f;
}

/* ------------------------------------------------------------------ costs */
typedef struct {
  int n_src, half_patch;
  float sigma_spatial, sigma_color, census_weight, smooth_weight, geom_weight;
  int top_k;
  float depth_min, depth_max;
} acm_params;

/* The tap loop is compiled twice, with and without the FMA instruction set,
 * and the loader picks the clone the host runs; fmaf rounds once either
 * way, so both give the same bits (a library call without FMA). */
#if defined(__GNUC__) && defined(__x86_64__) && !defined(__clang__)
__attribute__((target_clones("fma", "default")))
#endif
static float acm_ncc_at_stride(const acm_img* ref, const acm_img* src, float ref_center,
                               float src_center, float scx, float scy, int cx, int cy, int hp,
                               float stride, float ax, float ay, float bx, float by, float sf,
                               float cf) {
  float sw = 0.0f, sr = 0.0f, ss = 0.0f, srr = 0.0f, sss = 0.0f, srs = 0.0f;
  for (int iy = -hp; iy <= hp; ++iy)
    for (int ix = -hp; ix <= hp; ++ix) {
      const float fdx = stride * (float)ix, fdy = stride * (float)iy;
      const float rx = (float)cx + fdx, ry = (float)cy + fdy;
      const float rv = acm_sample(ref, rx + 0.5f, ry + 0.5f);
      const float sx = fmaf(bx, fdy, fmaf(ax, fdx, scx));
      const float sy = fmaf(by, fdy, fmaf(ay, fdx, scy));
      const float sv = acm_sample(src, sx + 0.5f, sy + 0.5f);
      const float dist2 = fmaf(fdy, fdy, fdx * fdx);
      const float r = rv - ref_center;
      const float w = acm_exp(fmaf(r * r, cf, dist2 * sf));
      const float s = sv - src_center;
      const float wr = w * r, ws = w * s;
      sr += wr;
      ss += ws;
      srr = fmaf(wr, r, srr);
      sss = fmaf(ws, s, sss);
      srs = fmaf(wr, s, srs);
      sw += w;
    }
  if (sw < 1e-6f) return -1.0f;
  const float inv = 1.0f / sw;
  const float mr = sr * inv, ms = ss * inv;
  const float vr = srr * inv - mr * mr;
  const float vs = sss * inv - ms * ms;
  if (vr < 1.5e-10f || vs < 1.5e-10f) return -1.0f;
  const float cov = srs * inv - mr * ms;
  return cov / sqrtf(vr * vs);
}

static float acm_ncc_multiscale(const acm_img* ref, const acm_img* src, float rc, float sc,
                                float scx, float scy, int cx, int cy, int hp, float ax, float ay,
                                float bx, float by, float sf, float cf) {
  static const float strides[3] = {1.0f, 2.0f, 3.0f};
  float best = -1.0f;
  int textureless = 0;
  for (int s = 0; s < 3; ++s) {
    float ncc = acm_ncc_at_stride(ref, src, rc, sc, scx, scy, cx, cy, hp, strides[s], ax, ay, bx,
                                  by, sf, cf);
    if (s == 0 && ncc < -0.5f) textureless = 1;
    if (textureless && ncc > 0.0f) ncc = 0.0f;
    if (ncc > best) best = ncc;
    if (best > 0.1f) return best;
  }
  return best;
}

static float acm_census(const acm_img* ref, const acm_img* src, float rc, float sc, int cx,
                        int cy, float scx, float scy, float ax, float ay, float bx, float by) {
  uint32_t rcen = 0, scen = 0;
  int bit = 0;
  for (int dy = -2; dy <= 2; ++dy)
    for (int dx = -2; dx <= 2; ++dx) {
      if (dx == 0 && dy == 0) continue;
      const float rv = acm_sample(ref, (float)(cx + dx) + 0.5f, (float)(cy + dy) + 0.5f);
      const float sx = (scx + ax * (float)dx) + bx * (float)dy;
      const float sy = (scy + ay * (float)dx) + by * (float)dy;
      const float sv = acm_sample(src, sx + 0.5f, sy + 0.5f);
      if (rv > rc) rcen |= 1u << bit;
      if (sv > sc) scen |= 1u << bit;
      ++bit;
    }
  const int ham = __builtin_popcount(rcen ^ scen);
  if (__builtin_popcount(rcen) < 3 && __builtin_popcount(scen) < 3) return 1.0f;
  return (float)ham / 24.0f;
}

static float acm_smoothstep(float e0, float e1, float x) {
  const float t = acm_clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return (t * t) * (3.0f - 2.0f * t);
}

static float acm_single_cost(const acm_img* ref, const acm_img* src, const acm_cam* sc,
                             const float* cw, const float* wdx, const float* wdy, float rc, int cx,
                             int cy, const acm_params* P, float sf, float cf) {
  float p[3], pdx[3], pdy[3];
  acm_project(sc, cw, p);
  if (p[2] < 1e-6f) return 2.0f;
  const float scx = p[0] / p[2], scy = p[1] / p[2];
  acm_project(sc, wdx, pdx);
  acm_project(sc, wdy, pdy);
  if (pdx[2] < 1e-6f || pdy[2] < 1e-6f) return 2.0f;
  const float ax = pdx[0] / pdx[2] - scx, ay = pdx[1] / pdx[2] - scy;
  const float bx = pdy[0] / pdy[2] - scx, by = pdy[1] / pdy[2] - scy;
  const float scen = acm_sample(src, scx + 0.5f, scy + 0.5f);
  const float ncc =
      acm_ncc_multiscale(ref, src, rc, scen, scx, scy, cx, cy, P->half_patch, ax, ay, bx, by, sf, cf);
  if (ncc <= -0.5f) {
    if (P->census_weight > 1e-6f) return acm_census(ref, src, rc, scen, cx, cy, scx, scy, ax, ay, bx, by);
    return 2.0f;
  }
  const float nc = 1.0f - ncc;
  if (P->census_weight < 1e-6f) return nc;
  const float t = acm_smoothstep(0.1f, 0.6f, nc);
  const float blend = P->census_weight * t;
  if (blend < 1e-4f) return nc;
  const float cen = acm_census(ref, src, rc, scen, cx, cy, scx, scy, ax, ay, bx, by);
  return (1.0f - blend) * nc + blend * cen;
}

typedef struct {
  const acm_img* imgs; /* [0] reference, [1 + i] source i */
  const acm_cam* cams;
  int W, H;
} acm_scene;

static void acm_cost_vector(const acm_scene* S, const acm_params* P, int x, int y,
                            const float* plane, float* out) {
  const acm_cam* c0 = &S->cams[0];
  const float depth = acm_depth_from_plane(c0, (float)x, (float)y, plane);
  if (depth <= 0.0f) {
    for (int i = 0; i < P->n_src; ++i) out[i] = 2.0f;
    return;
  }
  const float ddx = acm_depth_from_plane(c0, (float)(x + 1), (float)y, plane);
  const float ddy = acm_depth_from_plane(c0, (float)x, (float)(y + 1), plane);
  if (ddx <= 0.0f || ddy <= 0.0f) {
    for (int i = 0; i < P->n_src; ++i) out[i] = 2.0f;
    return;
  }
  float cw[3], wdx[3], wdy[3];
  acm_backproject(c0, (float)x, (float)y, depth, cw);
  acm_backproject(c0, (float)(x + 1), (float)y, ddx, wdx);
  acm_backproject(c0, (float)x, (float)(y + 1), ddy, wdy);
  const float rc = acm_sample(&S->imgs[0], (float)x + 0.5f, (float)y + 0.5f);
  const float sf = -1.0f / (2.0f * P->sigma_spatial * P->sigma_spatial);
  const float cf = -1.0f / (2.0f * P->sigma_color * P->sigma_color);
  for (int i = 0; i < P->n_src; ++i)
    out[i] = acm_single_cost(&S->imgs[0], &S->imgs[1 + i], &S->cams[1 + i], cw, wdx, wdy, rc, x,
                             y, P, sf, cf);
}

static float acm_initial_cost(const acm_scene* S, const acm_params* P, int x, int y,
                              const float* plane, uint32_t* sel) {
  float cv[ACM_MAX_SRC], cc[ACM_MAX_SRC];
  for (int i = 0; i < ACM_MAX_SRC; ++i) cv[i] = cc[i] = 2.0f;
  acm_cost_vector(S, P, x, y, plane, cv);
  int nv = 0;
  for (int i = 0; i < P->n_src; ++i) {
    cc[i] = cv[i];
    if (cv[i] < 2.0f) ++nv;
  }
  for (int i = 1; i < P->n_src; ++i) {
    const float tmp = cv[i];
    int j = i;
    for (; j >= 1 && tmp < cv[j - 1]; --j) cv[j] = cv[j - 1];
    cv[j] = tmp;
  }
  *sel = 0;
  int k = P->top_k < nv ? P->top_k : nv;
  if (P->n_src < k) k = P->n_src;
  if (k <= 0) return 2.0f;
  float total = 0.0f;
  for (int i = 0; i < k; ++i) total += cv[i];
  const float thr = cv[k - 1];
  for (int i = 0; i < P->n_src; ++i)
    if (cc[i] <= thr) *sel |= 1u << i;
  return total / (float)k;
}

static float acm_smoothness(const float* planes, const acm_cam* c, const float* cur, int x, int y,
                            int W, int H) {
  const float cd = acm_depth_from_plane(c, (float)x, (float)y, cur);
  if (cd <= 0.0f) return 0.0f;
  float cn[3] = {cur[0], cur[1], cur[2]};
  acm_normalize(cn);
  const float sig = 0.02f;
  static const int dxs[4] = {-1, 1, 0, 0}, dys[4] = {0, 0, -1, 1};
  float tw = 0.0f, tc = 0.0f;
  for (int k = 0; k < 4; ++k) {
    const int nx = x + dxs[k], ny = y + dys[k];
    if (nx < 0 || nx >= W || ny < 0 || ny >= H) continue;
    const float* nb = planes + 4 * ((size_t)ny * W + nx);
    const float nd = acm_depth_from_plane(c, (float)nx, (float)ny, nb);
    if (nd <= 0.0f) continue;
    const float rel = fabsf(cd - nd) / cd;
    const float w = acm_exp(-rel * rel / (2.0f * sig * sig));
    float nn[3] = {nb[0], nb[1], nb[2]};
    acm_normalize(nn);
    const float ncost = 1.0f - ((cn[0] * nn[0] + cn[1] * nn[1]) + cn[2] * nn[2]);
    const float pred = acm_depth_from_plane(c, (float)nx, (float)ny, cur);
    const float dev = pred > 0.0f ? fabsf(nd - pred) / cd : 0.0f;
    const float cost = 0.5f * acm_clampf(ncost, 0.0f, 1.0f) + 0.5f * acm_clampf(dev * 10.0f, 0.0f, 1.0f);
    tc += w * cost;
    tw += w;
  }
  if (tw < 1e-6f) return 0.0f;
  return tc / tw;
}

/* Previous-level depths of the sources (geometric consistency): [16][H][W]
 * at the current level's size, and which sources have one. */
typedef struct {
  const float* depths;
  uint32_t mask;
  const float* prior_planes; /* [H][W][4] SfM planar prior, or NULL */
  const uint32_t* prior_mask;
} acm_prev;

/* compute_geom_consistency_cost (opencl_kernels.h:945-990): the forward-
 * backward reprojection error through the source's previous depth, at most
 * 5 px. */
static float acm_geom_cost(const acm_cam* rc, const acm_cam* sc, const float* plane, int px,
                           int py, const float* prev, int W, int H) {
  const float maxc = 5.0f;
  const float depth = acm_depth_from_plane(rc, (float)px, (float)py, plane);
  if (depth <= 0.0f) return maxc;
  float w[3], p[3];
  acm_backproject(rc, (float)px, (float)py, depth, w);
  acm_project(sc, w, p);
  if (p[2] < 1e-6f) return maxc;
  const float sx = p[0] / p[2], sy = p[1] / p[2];
  if (sx < 0.0f || sx >= (float)W || sy < 0.0f || sy >= (float)H) return maxc;
  const int ix = acm_clampi((int)(sx + 0.5f), W), iy = acm_clampi((int)(sy + 0.5f), H);
  const float sd = prev[(size_t)iy * W + ix];
  if (sd <= 0.0f) return maxc;
  float sw[3], rp[3];
  acm_backproject(sc, sx, sy, sd, sw);
  acm_project(rc, sw, rp);
  if (rp[2] < 1e-6f) return maxc;
  const float bx = rp[0] / rp[2], by = rp[1] / rp[2];
  const float dx = (float)px - bx, dy = (float)py - by;
  const float e = sqrtf(dx * dx + dy * dy);
  return e < maxc ? e : maxc;
}

/* compute_weighted_cost_geom (opencl_kernels.h:1017-1045). */
static float acm_weighted(const float* cv, const float* vw, float norm, int n_src, float geom_w,
                          const acm_cam* cams, const float* plane, int x, int y,
                          const acm_prev* prev, int W, int H) {
  if (norm < 1e-6f) return 2.0f;
  float total = 0.0f;
  for (int i = 0; i < n_src; ++i)
    if (vw[i] > 0.0f) {
      float geom = 0.0f;
      if (geom_w > 0.0f && (prev->mask & (1u << i)))
        geom = acm_geom_cost(&cams[0], &cams[i + 1], plane, x, y,
                             prev->depths + (size_t)i * W * H, W, H);
      total += vw[i] * (cv[i] + geom_w * geom);
    }
  return total / norm;
}

/* ------------------------------------------------------------------ state */
typedef struct {
  float* planes; /* [H][W][4] */
  float* costs;  /* [H][W] */
  uint32_t* rs;  /* [H][W][2] */
  uint32_t* sel; /* [H][W] */
} acm_state;

static void acm_random_init(const acm_scene* S, const acm_params* P, acm_state* st) {
  const int W = S->W, H = S->H;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const int idx = y * W + x;
      uint32_t s[2] = {(uint32_t)idx * 1099087573u + 2654435769u,
                       (uint32_t)idx * 2246822519u + 13u};
      const uint32_t key = (uint32_t)(idx + 7919);
      const float lmin = acm_log(P->depth_min > 1e-6f ? P->depth_min : 1e-6f);
      const float lmax = acm_log(P->depth_max > 1e-5f ? P->depth_max : 1e-5f);
      const float depth = acm_exp(lmin + acm_rand(s, key) * (lmax - lmin));
      float n[3];
      n[0] = acm_rand(s, key + 3u) * 2.0f - 1.0f;
      n[1] = acm_rand(s, key + 5u) * 2.0f - 1.0f;
      n[2] = -1.0f;
      acm_normalize(n);
      float* pl = st->planes + 4 * (size_t)idx;
      acm_plane_from_depth_normal(&S->cams[0], (float)x, (float)y, depth, n, pl);
      st->rs[2 * idx] = s[0];
      st->rs[2 * idx + 1] = s[1];
      uint32_t sel = 0;
      st->costs[idx] = acm_initial_cost(S, P, x, y, pl, &sel);
      st->sel[idx] = sel;
    }
}

static void acm_pm_pixel(const acm_scene* S, const acm_params* P, acm_state* st, int x, int y,
                         int iteration, const acm_prev* prev) {
  const int W = S->W, H = S->H, npix = W * H;
  const int idx = y * W + x;
  const acm_cam* c0 = &S->cams[0];
  uint32_t s[2] = {st->rs[2 * idx], st->rs[2 * idx + 1]};
  const uint32_t key = (uint32_t)(idx + iteration * 7919 + 42);
  const int n_src = P->n_src;
  int pos[8], flags[8];
  float ca[8 * ACM_MAX_SRC];
  for (int i = 0; i < 8; ++i) {
    pos[i] = idx;
    flags[i] = 0;
  }
  for (int i = 0; i < 8 * ACM_MAX_SRC; ++i) ca[i] = 2.0f;
  const float* C = st->costs;
#define ACM_PICK(slot, cond, base_expr, LOOP)         \
  if (cond) {                                          \
    const int base = (base_expr);                      \
    float bc = C[base];                                \
    int bp = base;                                     \
    LOOP                                               \
    pos[slot] = bp;                                    \
    flags[slot] = 1;                                   \
    acm_cost_vector(S, P, x, y, st->planes + 4 * (size_t)bp, &ca[(slot) * ACM_MAX_SRC]); \
  }
#define ACM_TRY(pp_expr)                         \
  {                                              \
    const int pp = (pp_expr);                    \
    if (pp >= 0 && pp < npix && C[pp] < bc) {    \
      bc = C[pp];                                \
      bp = pp;                                   \
    }                                            \
  }
  /* Far candidates: every second pixel from 3 to 23 away (1, 3, 5, 7). */
  ACM_PICK(1, y > 2, (y - 3) * W + x,
           for (int i = 1; i < 11; ++i) { const int yy = y - 3 - 2 * i; if (yy < 0) break; const int pp = yy * W + x; if (C[pp] < bc) { bc = C[pp]; bp = pp; } })
  ACM_PICK(3, y < H - 3, (y + 3) * W + x,
           for (int i = 1; i < 11; ++i) { const int yy = y + 3 + 2 * i; if (yy >= H) break; const int pp = yy * W + x; if (C[pp] < bc) { bc = C[pp]; bp = pp; } })
  ACM_PICK(5, x > 2, y * W + (x - 3),
           for (int i = 1; i < 11; ++i) { const int xx = x - 3 - 2 * i; if (xx < 0) break; const int pp = y * W + xx; if (C[pp] < bc) { bc = C[pp]; bp = pp; } })
  ACM_PICK(7, x < W - 3, y * W + (x + 3),
           for (int i = 1; i < 11; ++i) { const int xx = x + 3 + 2 * i; if (xx >= W) break; const int pp = y * W + xx; if (C[pp] < bc) { bc = C[pp]; bp = pp; } })
  /* Near candidates: the neighbour and a V of diagonals behind it (0, 2, 4, 6). */
  ACM_PICK(0, y > 0, (y - 1) * W + x,
           for (int i = 0; i < 3; ++i) { if (y > 1 + i && x > i) ACM_TRY((y - 2 - i) * W + (x - i - 1)) if (y > 1 + i && x < W - 1 - i) ACM_TRY((y - 2 - i) * W + (x + i + 1)) })
  ACM_PICK(2, y < H - 1, (y + 1) * W + x,
           for (int i = 0; i < 3; ++i) { if (y < H - 2 - i && x > i) ACM_TRY((y + 2 + i) * W + (x - i - 1)) if (y < H - 2 - i && x < W - 1 - i) ACM_TRY((y + 2 + i) * W + (x + i + 1)) })
  ACM_PICK(4, x > 0, y * W + (x - 1),
           for (int i = 0; i < 3; ++i) { if (x > 1 + i && y > i) ACM_TRY((y - i - 1) * W + (x - 2 - i)) if (x > 1 + i && y < H - 1 - i) ACM_TRY((y + i + 1) * W + (x - 2 - i)) })
  ACM_PICK(6, x < W - 1, y * W + (x + 1),
           for (int i = 0; i < 3; ++i) { if (x < W - 2 - i && y > i) ACM_TRY((y - i - 1) * W + (x + 2 + i)) if (x < W - 2 - i && y < H - 1 - i) ACM_TRY((y + i + 1) * W + (x + 2 + i)) })
#undef ACM_PICK
#undef ACM_TRY

  /* View selection priors from the four direct neighbours (last one wins). */
  float pri[ACM_MAX_SRC];
  for (int i = 0; i < ACM_MAX_SRC; ++i) pri[i] = 0.0f;
  const int npos[4] = {idx - W, idx + W, idx - 1, idx + 1};
  for (int i = 0; i < 4; ++i) {
    const int np = npos[i];
    if (flags[2 * i] && np >= 0 && np < npix) {
      const uint32_t sv = st->sel[np];
      for (int j = 0; j < n_src; ++j) pri[j] = (sv & (1u << j)) ? 0.9f : 0.1f;
    }
  }
  const float thr = 0.8f * acm_exp((float)(iteration * iteration) / (-90.0f));
  float prob[ACM_MAX_SRC];
  for (int i = 0; i < ACM_MAX_SRC; ++i) prob[i] = 0.0f;
  for (int i = 0; i < n_src; ++i) {
    float count = 0.0f, tw = 0.0f;
    int cfalse = 0;
    for (int j = 0; j < 8; ++j) {
      const float cv = ca[j * ACM_MAX_SRC + i];
      if (flags[j] && cv < thr) {
        tw += acm_exp(cv * cv / (-0.18f));
        count += 1.0f;
      }
      if (flags[j] && cv > 1.2f) ++cfalse;
    }
    if (count > 2.0f && cfalse < 3)
      prob[i] = tw / count;
    else if (cfalse < 3)
      prob[i] = acm_exp(thr * thr / (-0.32f));
    prob[i] *= pri[i];
  }
  { /* pdf to cdf */
    float sum = 0.0f;
    for (int i = 0; i < n_src; ++i) sum += prob[i];
    if (!(sum < 1e-12f)) {
      const float inv = 1.0f / sum;
      float cum = 0.0f;
      for (int i = 0; i < n_src; ++i) {
        cum += prob[i] * inv;
        prob[i] = cum;
      }
    }
  }
  float vw[ACM_MAX_SRC];
  for (int i = 0; i < ACM_MAX_SRC; ++i) vw[i] = 0.0f;
  for (int smp = 0; smp < 15; ++smp) {
    const float r = acm_rand(s, key + (uint32_t)smp * 997u) - 1e-7f;
    for (int j = 0; j < n_src; ++j)
      if (prob[j] > r) {
        vw[j] += 1.0f;
        break;
      }
  }
  uint32_t new_sel = 0;
  float norm = 0.0f;
  for (int i = 0; i < n_src; ++i)
    if (vw[i] > 0.0f) {
      new_sel |= 1u << i;
      norm += vw[i];
    }

  float fc[8];
  for (int i = 0; i < 8; ++i) {
    if (flags[i]) {
      const float* pl = st->planes + 4 * (size_t)pos[i];
      const float photo = acm_weighted(&ca[i * ACM_MAX_SRC], vw, norm, n_src, P->geom_weight,
                                       S->cams, pl, x, y, prev, W, H);
      fc[i] = P->smooth_weight > 1e-6f
                  ? photo + P->smooth_weight * acm_smoothness(st->planes, c0, pl, x, y, W, H)
                  : photo;
    } else {
      fc[i] = 2.0f;
    }
  }
  int best = 0;
  float bcost = fc[0];
  for (int i = 1; i < 8; ++i)
    if (fc[i] < bcost) {
      bcost = fc[i];
      best = i;
    }
  float cvn[ACM_MAX_SRC];
  for (int i = 0; i < ACM_MAX_SRC; ++i) cvn[i] = 2.0f;
  float* own = st->planes + 4 * (size_t)idx;
  acm_cost_vector(S, P, x, y, own, cvn);
  float cost_now = acm_weighted(cvn, vw, norm, n_src, P->geom_weight, S->cams, own, x, y, prev, W, H);
  if (P->smooth_weight > 1e-6f)
    cost_now += P->smooth_weight * acm_smoothness(st->planes, c0, own, x, y, W, H);
  st->costs[idx] = cost_now;
  float plane_now[4] = {own[0], own[1], own[2], own[3]};
  float depth_now = acm_depth_from_plane(c0, (float)x, (float)y, plane_now);

  if (flags[best] && bcost < cost_now) {
    const float* bp = st->planes + 4 * (size_t)pos[best];
    const float db = acm_depth_from_plane(c0, (float)x, (float)y, bp);
    if (db >= P->depth_min && db <= P->depth_max) {
      depth_now = db;
      memcpy(plane_now, bp, sizeof(plane_now));
      cost_now = bcost;
      st->sel[idx] = new_sel;
    }
  }

  /* Refinement: five combinations of random / perturbed depth and normal. */
  const float pert = 0.02f;
  float cur_n[3] = {plane_now[0], plane_now[1], plane_now[2]};
  acm_normalize(cur_n);
  const float PI_F = 3.14159274101257324f;
  /* The SfM planar prior (opencl_kernels.h:1660-1740) centres the random
   * hypothesis on its plane where it covers the pixel. */
  const int have_prior = prev->prior_mask && prev->prior_mask[idx] > 0u;
  float depth_prior = 0.0f, prior_n[3] = {0.0f, 0.0f, -1.0f};
  if (have_prior) {
    const float* pp = prev->prior_planes + 4 * (size_t)idx;
    depth_prior = acm_depth_from_plane(c0, (float)x, (float)y, pp);
    prior_n[0] = pp[0];
    prior_n[1] = pp[1];
    prior_n[2] = pp[2];
    acm_normalize(prior_n);
  }
  float depth_rand, nr[3];
  if (have_prior && depth_prior > 0.0f) {
    const float dsig = (P->depth_max - P->depth_min) / 32.0f;
    const float asig = PI_F * (5.0f / 180.0f);
    depth_rand = depth_prior - 3.0f * dsig + acm_rand(s, key + 503u) * 6.0f * dsig;
    depth_rand = acm_clampf(depth_rand, P->depth_min, P->depth_max);
    const float q1 = (acm_rand(s, key + 504u) - 0.5f) * asig;
    const float q2 = (acm_rand(s, key + 505u) - 0.5f) * asig;
    nr[0] = prior_n[0] + q1;
    nr[1] = prior_n[1] + q2;
    nr[2] = prior_n[2];
    acm_normalize(nr);
    if (nr[2] > 0.0f) nr[2] = -nr[2];
  } else {
    const float lmin = acm_log(P->depth_min > 1e-6f ? P->depth_min : 1e-6f);
    const float lmax = acm_log(P->depth_max > 1e-5f ? P->depth_max : 1e-5f);
    depth_rand = acm_exp(lmin + acm_rand(s, key + 503u) * (lmax - lmin));
    nr[0] = acm_rand(s, key + 504u) * 2.0f - 1.0f;
    nr[1] = acm_rand(s, key + 505u) * 2.0f - 1.0f;
    nr[2] = -1.0f;
    acm_normalize(nr);
  }
  const float dmn = (1.0f - pert) * depth_now, dmx = (1.0f + pert) * depth_now;
  float depth_pert = dmn + acm_rand(s, key + 510u) * (dmx - dmn);
  depth_pert = acm_clampf(depth_pert, P->depth_min, P->depth_max);
  const float pa1 = ((acm_rand(s, key + 520u) - 0.5f) * pert) * PI_F;
  const float pa2 = ((acm_rand(s, key + 521u) - 0.5f) * pert) * PI_F;
  float np_[3] = {cur_n[0] + pa1, cur_n[1] + pa2, cur_n[2]};
  acm_normalize(np_);
  if (np_[2] > 0.0f) np_[2] = -np_[2];
  const float ds[5] = {depth_rand, depth_now, depth_rand, depth_now, depth_pert};
  const float* ns[5] = {cur_n, nr, nr, np_, cur_n};
  for (int h = 0; h < 5; ++h) {
    float cand[4];
    acm_plane_from_depth_normal(c0, (float)x, (float)y, ds[h], ns[h], cand);
    float cv[ACM_MAX_SRC];
    for (int i = 0; i < ACM_MAX_SRC; ++i) cv[i] = 2.0f;
    acm_cost_vector(S, P, x, y, cand, cv);
    float tc = acm_weighted(cv, vw, norm, n_src, P->geom_weight, S->cams, cand, x, y, prev, W, H);
    if (P->smooth_weight > 1e-6f)
      tc += P->smooth_weight * acm_smoothness(st->planes, c0, cand, x, y, W, H);
    const float db = acm_depth_from_plane(c0, (float)x, (float)y, cand);
    if (db < P->depth_min || db > P->depth_max) continue;
    if (tc < cost_now) {
      depth_now = db;
      memcpy(plane_now, cand, sizeof(plane_now));
      cost_now = tc;
    }
  }
  memcpy(own, plane_now, sizeof(plane_now));
  st->costs[idx] = cost_now;
  st->rs[2 * idx] = s[0];
  st->rs[2 * idx + 1] = s[1];
}

static void acm_sort(float* d, int n) {
  for (int i = 1; i < n; ++i) {
    const float t = d[i];
    int j = i;
    for (; j >= 1 && t < d[j - 1]; --j) d[j] = d[j - 1];
    d[j] = t;
  }
}

static void acm_filter_pixel(const acm_scene* S, acm_state* st, int x, int y) {
  const int W = S->W, H = S->H;
  const int c = y * W + x;
  const acm_cam* c0 = &S->cams[0];
  if (st->costs[c] < 0.001f) return;
  float buf[21];
  int n = 0;
#define ACM_D(cond, dx, dy)                                                                  \
  if (cond) buf[n++] = acm_depth_from_plane(c0, (float)(x + (dx)), (float)(y + (dy)),         \
                                            st->planes + 4 * (size_t)(c + (dy) * W + (dx)));
  buf[n++] = acm_depth_from_plane(c0, (float)x, (float)y, st->planes + 4 * (size_t)c);
  ACM_D(y > 0, 0, -1)
  ACM_D(y > 2, 0, -3)
  ACM_D(y > 4, 0, -5)
  ACM_D(y < H - 1, 0, 1)
  ACM_D(y < H - 3, 0, 3)
  ACM_D(y < H - 5, 0, 5)
  ACM_D(x > 0, -1, 0)
  ACM_D(x > 2, -3, 0)
  ACM_D(x > 4, -5, 0)
  ACM_D(x < W - 1, 1, 0)
  ACM_D(x < W - 3, 3, 0)
  ACM_D(x < W - 5, 5, 0)
  ACM_D(y > 0 && x < W - 2, 2, -1)
  ACM_D(y < H - 1 && x < W - 2, 2, 1)
  ACM_D(y > 0 && x > 1, -2, -1)
  ACM_D(y < H - 1 && x > 1, -2, 1)
  ACM_D(x > 0 && y > 2, -1, -2)
  ACM_D(x < W - 1 && y > 2, 1, -2)
  ACM_D(x > 0 && y < H - 2, -1, 2)
  ACM_D(x < W - 1 && y < H - 2, 1, 2)
#undef ACM_D
  const float cd = buf[0];
  if (cd > 0.0f) {
    const float lo = cd * (1 - 0.15f), hi = cd * (1 + 0.15f);
    int m = 1;
    for (int i = 1; i < n; ++i)
      if (buf[i] > lo && buf[i] < hi) buf[m++] = buf[i];
    n = m;
  }
  acm_sort(buf, n);
  const int mid = n / 2;
  const float med = (n % 2 == 0) ? (buf[mid - 1] + buf[mid]) * 0.5f : buf[mid];
  if (med > 0.0f) {
    float* pl = st->planes + 4 * (size_t)c;
    float nn[3] = {pl[0], pl[1], pl[2]};
    acm_normalize(nn);
    acm_plane_from_depth_normal(c0, (float)x, (float)y, med, nn, pl);
  }
}

/* 5x5 median with replicated borders (cv::medianBlur on a float image). */
static float acm_median5(const float* d, int W, int H, int x, int y) {
  float v[25];
  int k = 0;
  for (int a = -2; a <= 2; ++a)
    for (int b = -2; b <= 2; ++b) v[k++] = d[(size_t)acm_clampi(y + a, H) * W + acm_clampi(x + b, W)];
  acm_sort(v, 25);
  return v[12];
}

/* acmmp_upsample (opencl_kernels.h:1828-1892) after UpsampleDepthNormal's
 * host part (estimator.cc:600-640): the coarse level's depth, normal and
 * cost become planes at the coarse pixel, each fine pixel takes its
 * nearest coarse plane re-anchored at itself (or a random plane where the
 * coarse depth is invalid); every cost is 2, every view unselected. */
static void acm_upsample(const acm_scene* S, const acm_params* P, acm_state* st,
                         const float* cd, const float* cn, int sw, int sh) {
  const int W = S->W, H = S->H;
  const acm_cam* c0 = &S->cams[0];
  float* sp = (float*)malloc(sizeof(float) * 4 * (size_t)sw * sh);
  const float fx = c0->K[0] * (float)sw / (float)W, fy = c0->K[4] * (float)sh / (float)H;
  const float cxs = c0->K[2] * (float)sw / (float)W, cys = c0->K[5] * (float)sh / (float)H;
  for (int y = 0; y < sh; ++y)
    for (int x = 0; x < sw; ++x) {
      const size_t i = (size_t)y * sw + x;
      const float d = cd[i];
      const float* n = cn + 3 * i;
      const float p0 = d * ((float)x - cxs) / fx, p1 = d * ((float)y - cys) / fy, p2 = d;
      sp[4 * i] = n[0];
      sp[4 * i + 1] = n[1];
      sp[4 * i + 2] = n[2];
      sp[4 * i + 3] = -((n[0] * p0 + n[1] * p1) + n[2] * p2);
    }
  const float scx = (float)sw / (float)W, scy = (float)sh / (float)H;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const int idx = y * W + x;
      uint32_t s[2] = {(uint32_t)idx * 1099087573u + 2654435769u,
                       (uint32_t)idx * 2246822519u + 13u};
      st->rs[2 * idx] = s[0];
      st->rs[2 * idx + 1] = s[1];
      const int sx = acm_clampi((int)((float)x * scx), sw), sy = acm_clampi((int)((float)y * scy), sh);
      const float* pl = sp + 4 * ((size_t)sy * sw + sx);
      float* out = st->planes + 4 * (size_t)idx;
      const float depth = acm_depth_from_plane(c0, (float)x, (float)y, pl);
      if (depth > 0.0f) {
        float n[3] = {pl[0], pl[1], pl[2]};
        acm_normalize(n);
        acm_plane_from_depth_normal(c0, (float)x, (float)y, depth, n, out);
      } else {
        const uint32_t key = (uint32_t)(idx + 7919);
        const float lmin = acm_log(P->depth_min > 1e-6f ? P->depth_min : 1e-6f);
        const float lmax = acm_log(P->depth_max > 1e-5f ? P->depth_max : 1e-5f);
        const float rd = acm_exp(lmin + acm_rand(s, key) * (lmax - lmin));
        float n[3];
        n[0] = acm_rand(s, key + 3u) * 2.0f - 1.0f;
        n[1] = acm_rand(s, key + 5u) * 2.0f - 1.0f;
        n[2] = -1.0f;
        acm_normalize(n);
        acm_plane_from_depth_normal(c0, (float)x, (float)y, rd, n, out);
        st->rs[2 * idx] = s[0];
        st->rs[2 * idx + 1] = s[1];
      }
      st->costs[idx] = 2.0f;
      st->sel[idx] = 0;
    }
  free(sp);
}

/* cv::resize(INTER_AREA) of an 8-bit image by an integer factor k that
 * divides both sizes (OpenCV's fast area path): the k x k block mean,
 * rounded half up for k = 2, else float(sum) * float(1/k^2) rounded to
 * nearest even. */
void or_resize_area_u8(const uint8_t* src, int W, int H, int k, uint8_t* dst) {
  const int w = W / k, h = H / k;
  const float inv = 1.0f / (float)(k * k);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      int sum = 0;
      for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) sum += src[(size_t)(k * y + a) * W + (k * x + b)];
      int v;
      if (k == 2)
        v = (sum + 2) >> 2;
      else
        v = (int)nearbyintf((float)sum * inv);
      dst[(size_t)y * w + x] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
    }
}

/* cv::resize(INTER_AREA) of an 8-bit image to (w, h) when the ratios are not
 * both integers (OpenCV's general area path): per axis a table of source
 * cells and float weights (the overlap of each source pixel with the
 * destination cell over the cell width), a horizontal pass per source row
 * and a vertical accumulation, all in float, rounded half to even. */
typedef struct {
  int di, si;
  float alpha;
} acm_area_tab;

static int acm_area_table(int ssize, int dsize, double scale, acm_area_tab* t) {
  int k = 0;
  for (int dx = 0; dx < dsize; ++dx) {
    const double fsx1 = dx * scale, fsx2 = fsx1 + scale;
    const double cell = scale < ssize - fsx1 ? scale : ssize - fsx1;
    int sx1 = (int)ceil(fsx1), sx2 = (int)floor(fsx2);
    if (sx2 > ssize - 1) sx2 = ssize - 1;
    if (sx1 > sx2) sx1 = sx2;
    if (sx1 - fsx1 > 1e-3) {
      t[k].di = dx;
      t[k].si = sx1 - 1;
      t[k++].alpha = (float)((sx1 - fsx1) / cell);
    }
    for (int sx = sx1; sx < sx2; ++sx) {
      t[k].di = dx;
      t[k].si = sx;
      t[k++].alpha = (float)(1.0 / cell);
    }
    if (fsx2 - sx2 > 1e-3) {
      double a = fsx2 - sx2 < 1.0 ? fsx2 - sx2 : 1.0;
      if (a > cell) a = cell;
      t[k].di = dx;
      t[k].si = sx2;
      t[k++].alpha = (float)(a / cell);
    }
  }
  return k;
}

void or_resize_area_general_u8(const uint8_t* src, int W, int H, uint8_t* dst, int w, int h) {
  const double sx = 1.0 / ((double)w / W), sy = 1.0 / ((double)h / H);
  acm_area_tab* xt = (acm_area_tab*)malloc(sizeof(acm_area_tab) * 2 * (size_t)(W + 2));
  acm_area_tab* yt = (acm_area_tab*)malloc(sizeof(acm_area_tab) * 2 * (size_t)(H + 2));
  float* buf = (float*)malloc(sizeof(float) * (size_t)w);
  float* sum = (float*)malloc(sizeof(float) * (size_t)w);
  const int nx = acm_area_table(W, w, sx, xt), ny = acm_area_table(H, h, sy, yt);
  int prev = -1;
  for (int j = 0; j < ny; ++j) {
    const int dy = yt[j].di;
    const float beta = yt[j].alpha;
    const uint8_t* S = src + (size_t)yt[j].si * W;
    for (int dx = 0; dx < w; ++dx) buf[dx] = 0.0f;
    for (int k = 0; k < nx; ++k) buf[xt[k].di] += (float)S[xt[k].si] * xt[k].alpha;
    if (dy != prev) {
      if (prev >= 0)
        for (int dx = 0; dx < w; ++dx) {
          const int v = (int)nearbyintf(sum[dx]);
          dst[(size_t)prev * w + dx] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
        }
      for (int dx = 0; dx < w; ++dx) sum[dx] = beta * buf[dx];
      prev = dy;
    } else {
      for (int dx = 0; dx < w; ++dx) sum[dx] += beta * buf[dx];
    }
  }
  if (prev >= 0)
    for (int dx = 0; dx < w; ++dx) {
      const int v = (int)nearbyintf(sum[dx]);
      dst[(size_t)prev * w + dx] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
    }
  free(xt);
  free(yt);
  free(buf);
  free(sum);
}

/* Bilinear resize of a float image with OpenCV's pixel-centre mapping
 * (f = (d + 0.5) src/dst - 0.5 in double, clamped to the border pixels),
 * FP32 weights 1 - f and f, the horizontal then the vertical blend, each
 * product and sum rounded by itself.  OpenCV's own INTER_LINEAR runs SIMD
 * arithmetic and differs from this in the last bits. */
void or_resize_linear_f32(const float* src, int w, int h, float* dst, int W, int H) {
  for (int y = 0; y < H; ++y) {
    double fyd = (y + 0.5) * ((double)h / H) - 0.5;
    int sy = (int)floor(fyd);
    float fy = (float)(fyd - sy);
    if (sy < 0) {
      sy = 0;
      fy = 0.0f;
    }
    if (sy >= h - 1) {
      sy = h - 1;
      fy = 0.0f;
    }
    const int sy1 = sy + 1 < h ? sy + 1 : h - 1;
    for (int x = 0; x < W; ++x) {
      double fxd = (x + 0.5) * ((double)w / W) - 0.5;
      int sx = (int)floor(fxd);
      float fx = (float)(fxd - sx);
      if (sx < 0) {
        sx = 0;
        fx = 0.0f;
      }
      if (sx >= w - 1) {
        sx = w - 1;
        fx = 0.0f;
      }
      const int sx1 = sx + 1 < w ? sx + 1 : w - 1;
      const float a0 = 1.0f - fx, b0 = 1.0f - fy;
      const float r0 = src[(size_t)sy * w + sx] * a0 + src[(size_t)sy * w + sx1] * fx;
      const float r1 = src[(size_t)sy1 * w + sx] * a0 + src[(size_t)sy1 * w + sx1] * fx;
      dst[(size_t)y * W + x] = r0 * b0 + r1 * fy;
    }
  }
}

/* One pyramid level of one reference view (RunLevel, estimator.cc:159-243):
 * images[0] the reference, images[1 .. n_src] sources, already at this
 * level's size (Ks scaled).  Initialised randomly, or from the coarse
 * level's result (cd, cn, cw x ch) when cd is not NULL.  prev_depths
 * [16][H][W] / prev_mask: the sources' previous-level depths for the
 * geometric term (NULL / 0 for none).  apply_median: the final readback.
 * out: depth, normal [H][W][3], cost, confidence. */
int or_acmmp_level(const float* const* images, const int* widths, const int* heights,
                   const double* const* Ks, const double* const* Rs, const double* const* ts,
                   int num_images, int iterations, int patch_size, float sigma_spatial,
                   float sigma_color, int top_k, float census_weight, float smooth_weight,
                   float geom_weight, float depth_min, float depth_max, const float* cd,
                   const float* cn, int cw, int ch, const float* prev_depths, uint32_t prev_mask,
                   const float* prior_planes, const uint32_t* prior_mask, int apply_median,
                   float* out_depth, float* out_normal, float* out_cost, float* out_conf) {
  if (num_images < 2) return -1;
  acm_params P;
  P.n_src = num_images - 1 < ACM_MAX_SRC ? num_images - 1 : ACM_MAX_SRC;
  P.half_patch = patch_size / 2;
  P.sigma_spatial = sigma_spatial;
  P.sigma_color = sigma_color;
  P.census_weight = census_weight;
  P.smooth_weight = smooth_weight;
  P.geom_weight = geom_weight;
  P.top_k = top_k;
  P.depth_min = depth_min;
  P.depth_max = depth_max;
  acm_img imgs[1 + ACM_MAX_SRC];
  acm_cam cams[1 + ACM_MAX_SRC];
  for (int i = 0; i <= P.n_src; ++i) {
    imgs[i].px = images[i];
    imgs[i].W = widths[i];
    imgs[i].H = heights[i];
    for (int k = 0; k < 9; ++k) {
      cams[i].K[k] = (float)Ks[i][k];
      cams[i].R[k] = (float)Rs[i][k];
    }
    for (int k = 0; k < 3; ++k) cams[i].t[k] = (float)ts[i][k];
  }
  const int W = widths[0], H = heights[0];
  const size_t npix = (size_t)W * H;
  acm_scene S = {imgs, cams, W, H};
  acm_state st;
  st.planes = (float*)calloc(4 * npix, sizeof(float));
  st.costs = (float*)calloc(npix, sizeof(float));
  st.rs = (uint32_t*)calloc(2 * npix, sizeof(uint32_t));
  st.sel = (uint32_t*)calloc(npix, sizeof(uint32_t));
  if (!st.planes || !st.costs || !st.rs || !st.sel) return -2;
  /* UploadPreviousDepths (estimator.cc:56-106) zeroes the mask without a
   * geometric weight. */
  acm_prev prev = {prev_depths, (prev_depths && geom_weight > 0.0f) ? prev_mask : 0u,
                   prior_planes, prior_planes ? prior_mask : NULL};
  if (cd)
    acm_upsample(&S, &P, &st, cd, cn, cw, ch);
  else
    acm_random_init(&S, &P, &st);
  for (int it = 0; it < iterations; ++it) {
    for (int colour = 0; colour < 2; ++colour)
      for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
          if (((x + y) & 1) == colour) acm_pm_pixel(&S, &P, &st, x, y, it, &prev);
    for (int colour = 0; colour < 2; ++colour)
      for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
          if (((x + y) & 1) == colour) acm_filter_pixel(&S, &st, x, y);
  }
  /* ReadBackResults (estimator.cc:941-1040). */
  for (size_t i = 0; i < npix; ++i) {
    out_depth[i] = 0.0f;
    out_normal[3 * i] = out_normal[3 * i + 1] = out_normal[3 * i + 2] = 0.0f;
    out_cost[i] = 0.0f;
    out_conf[i] = 0.0f;
  }
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const size_t i = (size_t)y * W + x;
      const float* p = st.planes + 4 * i;
      if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2]) || !isfinite(p[3])) continue;
      const float r0 = ((float)x - cams[0].K[2]) / cams[0].K[0];
      const float r1 = ((float)y - cams[0].K[5]) / cams[0].K[4];
      const float den = (p[0] * r0 + p[1] * r1) + p[2] * 1.0f;
      float depth = fabsf(den) > 1e-6f ? -p[3] / den : 0.0f;
      if (!isfinite(depth)) depth = 0.0f;
      if (depth > 0.0f && depth >= depth_min && depth <= depth_max) {
        out_depth[i] = depth;
        const float len = sqrtf((p[0] * p[0] + p[1] * p[1]) + p[2] * p[2]);
        if (len > 1e-6f)
          for (int k = 0; k < 3; ++k) out_normal[3 * i + k] = p[k] / len;
      }
      const float cst = st.costs[i];
      out_cost[i] = isfinite(cst) ? cst : 0.0f;
    }
  if (apply_median) {
    float* med = (float*)malloc(npix * sizeof(float));
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x) med[(size_t)y * W + x] = acm_median5(out_depth, W, H, x, y);
    for (size_t i = 0; i < npix; ++i) {
      const float d = out_depth[i], m = med[i];
      if (d > 0.0f && m > 0.0f && fabsf(d - m) / d > 0.10f) out_depth[i] = 0.0f;
    }
    free(med);
  }
  for (size_t i = 0; i < npix; ++i)
    if (out_depth[i] > 0.0f) out_conf[i] = 1.0f / (1.0f + expf((out_cost[i] - 0.5f) * 5.0f));
  free(st.planes);
  free(st.costs);
  free(st.rs);
  free(st.sel);
  return 0;
}

/* One reference view on one level: random initialisation, no previous
 * depths, the final readback. */
int or_acmmp_run(const float* const* images, const int* widths, const int* heights,
                 const double* const* Ks, const double* const* Rs, const double* const* ts,
                 int num_images, int iterations, int patch_size, float sigma_spatial,
                 float sigma_color, int top_k, float census_weight, float smooth_weight,
                 float geom_weight, float depth_min, float depth_max, float* out_depth,
                 float* out_normal, float* out_cost, float* out_conf) {
  return or_acmmp_level(images, widths, heights, Ks, Rs, ts, num_images, iterations, patch_size,
                        sigma_spatial, sigma_color, top_k, census_weight, smooth_weight,
                        geom_weight, depth_min, depth_max, NULL, NULL, 0, 0, NULL, 0, NULL, NULL,
                        1, out_depth, out_normal, out_cost, out_conf);
}

/* The random initialisation alone (planes [H][W][4], costs, selected views),
 * for tests of the first kernel. */
int or_acmmp_init(const float* const* images, const int* widths, const int* heights,
                  const double* const* Ks, const double* const* Rs, const double* const* ts,
                  int num_images, int patch_size, float sigma_spatial, float sigma_color,
                  int top_k, float census_weight, float depth_min, float depth_max,
                  float* planes, float* costs, uint32_t* sel) {
  if (num_images < 2) return -1;
  acm_params P;
  memset(&P, 0, sizeof(P));
  P.n_src = num_images - 1 < ACM_MAX_SRC ? num_images - 1 : ACM_MAX_SRC;
  P.half_patch = patch_size / 2;
  P.sigma_spatial = sigma_spatial;
  P.sigma_color = sigma_color;
  P.census_weight = census_weight;
  P.top_k = top_k;
  P.depth_min = depth_min;
  P.depth_max = depth_max;
  acm_img imgs[1 + ACM_MAX_SRC];
  acm_cam cams[1 + ACM_MAX_SRC];
  for (int i = 0; i <= P.n_src; ++i) {
    imgs[i].px = images[i];
    imgs[i].W = widths[i];
    imgs[i].H = heights[i];
    for (int k = 0; k < 9; ++k) {
      cams[i].K[k] = (float)Ks[i][k];
      cams[i].R[k] = (float)Rs[i][k];
    }
    for (int k = 0; k < 3; ++k) cams[i].t[k] = (float)ts[i][k];
  }
  const int W = widths[0], H = heights[0];
  const size_t npix = (size_t)W * H;
  acm_scene S = {imgs, cams, W, H};
  acm_state st;
  st.planes = planes;
  st.costs = costs;
  st.rs = (uint32_t*)calloc(2 * npix, sizeof(uint32_t));
  st.sel = sel;
  if (!st.rs) return -2;
  acm_random_init(&S, &P, &st);
  free(st.rs);
  return 0;
}

/* ComputeSfMPlanarPrior, first half (estimator.cc:683-728): the SfM points
 * (world, double) projected with the level's K (cast to float) and the
 * reference pose; those in front, in the depth range and inside the image
 * are kept.  uv [2N], depth [N], cam [3N]; returns the count. */
long or_acmmp_sfm_project(const double* pts, long n, const double* K, const double* R,
                          const double* t, int w, int h, float depth_min, float depth_max,
                          float* uv, float* depth, float* cam) {
  const float fx = (float)K[0], fy = (float)K[4], cx = (float)K[2], cy = (float)K[5];
  long m = 0;
  for (long i = 0; i < n; ++i) {
    const double* X = pts + 3 * i;
    double c[3];
    for (int r = 0; r < 3; ++r) c[r] = ((R[3 * r] * X[0] + R[3 * r + 1] * X[1]) + R[3 * r + 2] * X[2]) + t[r];
    if (c[2] <= 0.0) continue;
    const float d = (float)c[2];
    if (d < depth_min || d > depth_max) continue;
    const float u = (float)((double)fx * (c[0] / c[2]) + (double)cx);
    const float v = (float)((double)fy * (c[1] / c[2]) + (double)cy);
    if (u < 0.0f || u >= (float)w || v < 0.0f || v >= (float)h) continue;
    uv[2 * m] = u;
    uv[2 * m + 1] = v;
    depth[m] = d;
    cam[3 * m] = (float)c[0];
    cam[3 * m + 1] = (float)c[1];
    cam[3 * m + 2] = (float)c[2];
    ++m;
  }
  return m;
}

/* ComputeSfMPlanarPrior, second half (estimator.cc:740-940) over given
 * Delaunay triangles (ascending index triples, sorted): the integer-pixel
 * vertex lookup (last point wins), the depth-ratio and area gates, the
 * plane through the three camera points (unit cross-product normal, d >= 0),
 * the parametric rasterisation in order and the depth-range check.  planes
 * [H][W][4] (unset: 0, 0, -1, 0), mask [H][W].  Returns the masked count. */
long or_acmmp_sfm_prior(const float* uv, const float* depth, const float* cam, long m,
                        const int* tris, long n_tris, const double* K, int w, int h,
                        float depth_min, float depth_max, float* planes, uint32_t* mask) {
  const float fx = (float)K[0], fy = (float)K[4], cx = (float)K[2], cy = (float)K[5];
  const size_t npix = (size_t)w * h;
  for (size_t i = 0; i < npix; ++i) {
    planes[4 * i] = 0.0f;
    planes[4 * i + 1] = 0.0f;
    planes[4 * i + 2] = -1.0f;
    planes[4 * i + 3] = 0.0f;
    mask[i] = 0u;
  }
  if (m < 4) return 0;
  float* tp = (float*)malloc(sizeof(float) * 4 * (size_t)(n_tris + 1));
  int* tx = (int*)malloc(sizeof(int) * 6 * (size_t)(n_tris + 1));
  long kept = 0;
  for (long ti = 0; ti < n_tris; ++ti) {
    int px[3], py[3], src[3], ok = 1;
    for (int k = 0; k < 3; ++k) {
      const int v = tris[3 * ti + k];
      px[k] = (int)uv[2 * v];
      py[k] = (int)uv[2 * v + 1];
      if (px[k] < 0 || px[k] >= w || py[k] < 0 || py[k] >= h) ok = 0;
      src[k] = -1;
      for (long j = 0; j < m; ++j)
        if ((int)uv[2 * j + 1] == py[k] && (int)uv[2 * j] == px[k]) src[k] = (int)j;
      if (src[k] < 0) ok = 0;
    }
    if (!ok) continue;
    float dmin = depth[src[0]], dmax = depth[src[0]];
    for (int k = 1; k < 3; ++k) {
      if (depth[src[k]] < dmin) dmin = depth[src[k]];
      if (depth[src[k]] > dmax) dmax = depth[src[k]];
    }
    if (dmin > 0.0f && dmax / dmin > 1.5f) continue;
    const float ax = (float)(px[1] - px[0]), ay = (float)(py[1] - py[0]);
    const float bx = (float)(px[2] - px[0]), by = (float)(py[2] - py[0]);
    if (0.5f * fabsf(ax * by - ay * bx) > 20000.0f) continue;
    const float* P1 = cam + 3 * src[0];
    const float* P2 = cam + 3 * src[1];
    const float* P3 = cam + 3 * src[2];
    const float e1[3] = {P2[0] - P1[0], P2[1] - P1[1], P2[2] - P1[2]};
    const float e2[3] = {P3[0] - P1[0], P3[1] - P1[1], P3[2] - P1[2]};
    float nn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                   e1[0] * e2[1] - e1[1] * e2[0]};
    const float len = sqrtf((nn[0] * nn[0] + nn[1] * nn[1]) + nn[2] * nn[2]);
    if (!(len > 0.0f)) continue;
    for (int k = 0; k < 3; ++k) nn[k] = nn[k] / len;
    float d = -((nn[0] * P1[0] + nn[1] * P1[1]) + nn[2] * P1[2]);
    if (1.0f / sqrtf(1.0f + d * d) < 1e-8f) continue;
    if (d < 0.0f) {
      for (int k = 0; k < 3; ++k) nn[k] = -nn[k];
      d = -d;
    }
    float* pl = tp + 4 * kept;
    pl[0] = nn[0];
    pl[1] = nn[1];
    pl[2] = nn[2];
    pl[3] = d;
    for (int k = 0; k < 3; ++k) {
      tx[6 * kept + k] = px[k];
      tx[6 * kept + 3 + k] = py[k];
    }
    ++kept;
  }
  int* at = (int*)calloc(npix, sizeof(int));
  for (long ti = 0; ti < kept; ++ti) {
    const int* X = tx + 6 * ti;
    const int* Y = X + 3;
    const float l01 = hypotf((float)(X[0] - X[1]), (float)(Y[0] - Y[1]));
    const float l02 = hypotf((float)(X[0] - X[2]), (float)(Y[0] - Y[2]));
    const float l12 = hypotf((float)(X[1] - X[2]), (float)(Y[1] - Y[2]));
    float me = l01 > l02 ? l01 : l02;
    if (l12 > me) me = l12;
    if (me < 1.0f) continue;
    const float step = 1.0f / me;
    for (float p = 0.0f; p < 1.0f; p += step)
      for (float q = 0.0f; q < 1.0f - p; q += step) {
        const int xx = (int)(p * (float)X[0] + q * (float)X[1] + (1.0f - p - q) * (float)X[2]);
        const int yy = (int)(p * (float)Y[0] + q * (float)Y[1] + (1.0f - p - q) * (float)Y[2]);
        if (xx >= 0 && xx < w && yy >= 0 && yy < h) at[(size_t)yy * w + xx] = (int)ti + 1;
      }
  }
  long filled = 0;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const size_t i = (size_t)y * w + x;
      if (!at[i]) continue;
      const float* pl = tp + 4 * (at[i] - 1);
      const float r0 = ((float)x - cx) / fx, r1 = ((float)y - cy) / fy;
      const float den = (pl[0] * r0 + pl[1] * r1) + pl[2] * 1.0f;
      const float dd = fabsf(den) > 1e-6f ? -pl[3] / den : 0.0f;
      if (dd >= depth_min && dd <= depth_max) {
        for (int k = 0; k < 4; ++k) planes[4 * i + k] = pl[k];
        mask[i] = 1u;
        ++filled;
      }
    }
  free(at);
  free(tp);
  free(tx);
  return filled;
}
