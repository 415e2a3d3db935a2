// DepthmapClusterEstimator (cluster.h, cluster_estimator.cc:21-147) over the
// live path's PatchMatch estimator (estimator.h:33-135, estimator.cc:120-243,
// 473-558, 941-1040) and its kernels (opencl_kernels.h:44-1124, 1298-1826,
// 1828-2099): pyramid levels with upsampling and geometric consistency, and
// the SfM planar prior (estimator.cc:664-940).
//
// Per reference view and level: a random initialisation with top-k view
// selection (or, above the coarsest level, the coarser result upsampled),
// then per iteration a red and a black PatchMatch pass (8 propagation
// candidates, multi-hypothesis joint view selection, 5 refinement
// hypotheses; the matching cost is a bilateral NCC over strides 1, 2, 3
// with a census-transform fallback and blend) and a red and a black
// checkerboard median filter; then the readback (depth and normal from the
// planes, a 5x5 median rejection, a logistic confidence).
//
// The reference's float results depend on its OpenCL device
// (hardware-filtered image reads, exp/log/normalize precision,
// contraction).  This file fixes one arithmetic, the one the C oracle
// restates, and matches it bit for bit:
//   - FP32, every operation rounded by itself in the written order: the
//     file is compiled without FMA contraction (--fmad=false), and the
//     only fused multiply-adds are the __fmaf_rn written out in the NCC
//     tap, the bilinear blend and acm_exp (fmaf at the same places in the
//     oracle);
//   - acm_exp / acm_log below (Cody-Waite reduction, fixed polynomials);
//   - images as float(v) * float(1/255); linear, clamp-to-edge reads as the
//     OpenCL specification defines them, with exact fractions;
//   - normalize(v) = v / sqrt((x*x + y*y) + z*z).
// Images live in HBM as FP32 planes; every kernel is one thread per pixel
// (per pixel of the pass's colour), and the state (planes, costs, RNG
// states, selected views) stays on the device between the passes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "dense_b200.h"
#include "device_guard.h"

namespace {

thread_local std::string g_acm_error;

dn_status afail(dn_status s, const std::string& m) {
  g_acm_error = m;
  return s;
}

#define ACHECK(cond, msg) \
  do {                    \
    if (!(cond)) return afail(DN_INVALID_ARG, msg); \
  } while (0)
#define ACUDA(expr)                                                        \
  do {                                                                     \
    cudaError_t e_ = (expr);                                               \
    if (e_ != cudaSuccess) {                                               \
      return afail(e_ == cudaErrorMemoryAllocation ? DN_OUT_OF_MEMORY      \
                                                   : DN_DEVICE_ERROR,      \
                   cudaGetErrorString(e_));                                \
    }                                                                      \
  } while (0)

constexpr int kMaxSrc = 16;  // MAX_SOURCES

struct AImg {
  const float* px;
  int W, H;
};
struct ACam {
  float K[9], R[9], t[3];
};
struct AScene {
  AImg img[1 + kMaxSrc];  // [0] reference
  ACam cam[1 + kMaxSrc];
  int W, H, n_src, half_patch, top_k;
  float sigma_spatial, sigma_color, census_weight, smooth_weight, geom_weight;
  float depth_min, depth_max;
  const float* prev;   // [16][H][W] previous-level source depths, or null
  unsigned prev_mask;  // sources with a previous depth (0 without a geometric weight)
  const float4* prior_planes;  // SfM planar prior per pixel, or null
  const unsigned* prior_mask;  // pixels the prior covers
};
struct AState {
  float4* planes;  // (nx, ny, nz, d): n . X + d = 0 in the camera frame
  float* costs;
  uint2* rs;
  unsigned* sel;
};

// ------------------------------------------------------------ arithmetic
__device__ inline float acm_ldexp(float p, int n) {
  const int n1 = n / 2, n2 = n - n1;
  if (n1 < -126 || n2 < -126 || n1 > 127 || n2 > 127) return n < 0 ? 0.0f : INFINITY;
  return (p * __int_as_float((n1 + 127) << 23)) * __int_as_float((n2 + 127) << 23);
}

// e^x: n = round(x log2 e), r = x - n ln2 in two parts, degree-7 Taylor
// in Horner form; the reduction and the Horner steps are fused
// multiply-adds.
__device__ inline float acm_exp(float x) {
  if (x != x) return x;
  if (x > 88.72283f) return INFINITY;
  if (x < -103.97208f) return 0.0f;
  const float t = x * 1.44269502f;
  const float nf = floorf(t + 0.5f);
  const int n = (int)nf;
  const float r = __fmaf_rn(-nf, 1.42860677e-06f, __fmaf_rn(-nf, 0.693145752f, x));
  float p = 1.98412701e-04f;
  p = __fmaf_rn(p, r, 1.38888892e-03f);
  p = __fmaf_rn(p, r, 8.33333377e-03f);
  p = __fmaf_rn(p, r, 4.16666679e-02f);
  p = __fmaf_rn(p, r, 1.66666672e-01f);
  p = __fmaf_rn(p, r, 0.5f);
  p = __fmaf_rn(p, r, 1.0f);
  p = __fmaf_rn(p, r, 1.0f);
  return acm_ldexp(p, n);
}

// ln x: x = m 2^e, m in [sqrt(1/2), sqrt(2)), 2 atanh((m - 1) / (m + 1)).
__device__ inline float acm_log(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  unsigned u = __float_as_uint(x);
  int e = 0;
  if (u < 0x00800000u) {
    u = __float_as_uint(x * 16777216.0f);
    e = -24;
  }
  e += (int)(u >> 23) - 127;
  float m = __uint_as_float((u & 0x007FFFFFu) | 0x3F800000u);
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

__device__ inline float3 acm_normalize(float3 v) {
  const float len = sqrtf((v.x * v.x + v.y * v.y) + v.z * v.z);
  if (len == 0.0f) return v;
  return make_float3(v.x / len, v.y / len, v.z / len);
}

__device__ inline float acm_clamp(float x, float lo, float hi) {
  const float m = x > lo ? x : lo;
  return m < hi ? m : hi;
}

__device__ inline int clampi(int i, int n) { return i < 0 ? 0 : (i >= n ? n - 1 : i); }

// The bilinear blend ((w00 t00 + w10 t10) + w01 t01) + w11 t11 of the
// texels at fractions (a, b), the last three terms as fused multiply-adds.
__device__ inline float acm_lerp4(float a, float b, float t00, float t10, float t01, float t11) {
  const float ia = 1.0f - a, ib = 1.0f - b;
  return __fmaf_rn(a * b, t11, __fmaf_rn(ia * b, t01, __fmaf_rn(a * ib, t10, (ia * ib) * t00)));
}

// read_imagef(linear, clamp-to-edge) at unnormalised (u, v).
__device__ inline float acm_sample(const AImg& im, float u, float v) {
  float xm = u - 0.5f, ym = v - 0.5f;
  if (!(xm >= -16.0f)) xm = -16.0f;
  if (!(xm <= (float)im.W + 16.0f)) xm = (float)im.W + 16.0f;
  if (!(ym >= -16.0f)) ym = -16.0f;
  if (!(ym <= (float)im.H + 16.0f)) ym = (float)im.H + 16.0f;
  const float fx = floorf(xm), fy = floorf(ym);
  const float a = xm - fx, b = ym - fy;
  const int i0 = (int)fx, j0 = (int)fy;
  const int xa = clampi(i0, im.W), xb = clampi(i0 + 1, im.W);
  const int ya = clampi(j0, im.H), yb = clampi(j0 + 1, im.H);
  const float* p = im.px;
  const float t00 = __ldg(p + (size_t)ya * im.W + xa), t10 = __ldg(p + (size_t)ya * im.W + xb);
  const float t01 = __ldg(p + (size_t)yb * im.W + xa), t11 = __ldg(p + (size_t)yb * im.W + xb);
  return acm_lerp4(a, b, t00, t10, t01, t11);
}

// The same read at an integer texel (x + 0.5, y + 0.5): the fractions are
// 0, so the formula above returns the (clamped) texel itself exactly.
__device__ inline float acm_texel(const AImg& im, int x, int y) {
  return __ldg(im.px + (size_t)clampi(y, im.H) * im.W + clampi(x, im.W));
}

// The read of acm_sample for a (u, v) known to satisfy 1 <= u - 0.5 and
// u - 0.5 <= W - 2 (likewise v): no clamp changes anything there.
__device__ inline float acm_sample_inside(const AImg& im, float u, float v) {
  const float xm = u - 0.5f, ym = v - 0.5f;
  const float fx = floorf(xm), fy = floorf(ym);
  const float a = xm - fx, b = ym - fy;
  const float* p = im.px + (size_t)(int)fy * im.W + (int)fx;
  const float t00 = __ldg(p), t10 = __ldg(p + 1);
  const float t01 = __ldg(p + im.W), t11 = __ldg(p + im.W + 1);
  return acm_lerp4(a, b, t00, t10, t01, t11);
}

__device__ inline float3 acm_project(const ACam& c, float3 X) {
  const float x0 = ((c.R[0] * X.x + c.R[1] * X.y) + c.R[2] * X.z) + c.t[0];
  const float x1 = ((c.R[3] * X.x + c.R[4] * X.y) + c.R[5] * X.z) + c.t[1];
  const float x2 = ((c.R[6] * X.x + c.R[7] * X.y) + c.R[8] * X.z) + c.t[2];
  return make_float3((c.K[0] * x0 + c.K[1] * x1) + c.K[2] * x2,
                     (c.K[3] * x0 + c.K[4] * x1) + c.K[5] * x2,
                     (c.K[6] * x0 + c.K[7] * x1) + c.K[8] * x2);
}

__device__ inline float3 acm_backproject(const ACam& c, float x, float y, float depth) {
  const float px = depth * (x - c.K[2]) / c.K[0];
  const float py = depth * (y - c.K[5]) / c.K[4];
  const float d0 = px - c.t[0], d1 = py - c.t[1], d2 = depth - c.t[2];
  return make_float3((c.R[0] * d0 + c.R[3] * d1) + c.R[6] * d2,
                     (c.R[1] * d0 + c.R[4] * d1) + c.R[7] * d2,
                     (c.R[2] * d0 + c.R[5] * d1) + c.R[8] * d2);
}

__device__ inline float acm_depth(const ACam& c, float x, float y, float4 pl) {
  const float den = (pl.x * (x - c.K[2]) / c.K[0] + pl.y * (y - c.K[5]) / c.K[4]) + pl.z;
  if (fabsf(den) < 1e-6f) return 0.0f;
  return -pl.w / den;
}

__device__ inline float4 acm_plane(const ACam& c, float x, float y, float depth, float3 n) {
  const float p0 = depth * (x - c.K[2]) / c.K[0];
  const float p1 = depth * (y - c.K[5]) / c.K[4];
  return make_float4(n.x, n.y, n.z, -((n.x * p0 + n.y * p1) + n.z * depth));
}

__device__ inline float acm_rand(uint2& st, unsigned key) {
#pragma unroll
  for (unsigned i = 0; i < 4; ++i) {
    const unsigned k = key + i * 0x9E3779B9u;
    const unsigned lo = st.x * 0xD256D193u, hi = __umulhi(st.x, 0xD256D193u);
    st = make_uint2(st.y ^ k ^ hi, lo);
  }
  return (float)st.x / 4294967296.0f;
}

// ------------------------------------------------------------------ costs
__device__ float ncc_at_stride(const AImg& ref, const AImg& src, float rc, float sc, float scx,
                               float scy, int cx, int cy, int hp, float stride, float ax,
                               float ay, float bx, float by, float sf, float cf) {
  float sw = 0.0f, sr = 0.0f, ss = 0.0f, srr = 0.0f, sss = 0.0f, srs = 0.0f;
  // The warped patch is affine: if its corners lie at least a texel inside
  // the source (with a margin for the rounding of the inner taps), no tap
  // is clamped and the reads skip the clamps.
  const float e = stride * (float)hp;
  const float ex = fabsf(ax) * e + fabsf(bx) * e, ey = fabsf(ay) * e + fabsf(by) * e;
  const bool inside = scx - ex >= 1.5f && scx + ex <= (float)src.W - 3.5f &&
                      scy - ey >= 1.5f && scy + ey <= (float)src.H - 3.5f;
  const int istride = (int)stride;
  for (int iy = -hp; iy <= hp; ++iy)
    for (int ix = -hp; ix <= hp; ++ix) {
      const float fdx = stride * (float)ix, fdy = stride * (float)iy;
      // Reference taps sit on integer texels (integer strides).
      const float rv = acm_texel(ref, cx + istride * ix, cy + istride * iy);
      const float sx = __fmaf_rn(bx, fdy, __fmaf_rn(ax, fdx, scx));
      const float sy = __fmaf_rn(by, fdy, __fmaf_rn(ay, fdx, scy));
      const float sv = inside ? acm_sample_inside(src, sx + 0.5f, sy + 0.5f)
                              : acm_sample(src, sx + 0.5f, sy + 0.5f);
      const float dist2 = __fmaf_rn(fdy, fdy, fdx * fdx);
      const float r = rv - rc;
      const float w = acm_exp(__fmaf_rn(r * r, cf, dist2 * sf));
      const float s = sv - sc;
      const float wr = w * r, ws = w * s;
      sr += wr;
      ss += ws;
      srr = __fmaf_rn(wr, r, srr);
      sss = __fmaf_rn(ws, s, sss);
      srs = __fmaf_rn(wr, s, srs);
      sw += w;
    }
  if (sw < 1e-6f) return -1.0f;
  const float inv = 1.0f / sw;
  const float mr = sr * inv, ms = ss * inv;
  const float vr = srr * inv - mr * mr, vs = sss * inv - ms * ms;
  if (vr < 1.5e-10f || vs < 1.5e-10f) return -1.0f;
  return (srs * inv - mr * ms) / sqrtf(vr * vs);
}

__device__ float ncc_multiscale(const AImg& ref, const AImg& src, float rc, float sc, float scx,
                                float scy, int cx, int cy, int hp, float ax, float ay, float bx,
                                float by, float sf, float cf) {
  float best = -1.0f;
  bool textureless = false;
  for (int s = 0; s < 3; ++s) {
    float ncc = ncc_at_stride(ref, src, rc, sc, scx, scy, cx, cy, hp, (float)(s + 1), ax, ay, bx,
                              by, sf, cf);
    if (s == 0 && ncc < -0.5f) textureless = true;
    if (textureless && ncc > 0.0f) ncc = 0.0f;
    if (ncc > best) best = ncc;
    if (best > 0.1f) return best;
  }
  return best;
}

__device__ float census(const AImg& ref, const AImg& src, float rc, float sc, int cx, int cy,
                        float scx, float scy, float ax, float ay, float bx, float by) {
  unsigned rb = 0, sb = 0;
  int bit = 0;
  for (int dy = -2; dy <= 2; ++dy)
    for (int dx = -2; dx <= 2; ++dx) {
      if (dx == 0 && dy == 0) continue;
      const float rv = acm_texel(ref, cx + dx, cy + dy);
      const float sx = (scx + ax * (float)dx) + bx * (float)dy;
      const float sy = (scy + ay * (float)dx) + by * (float)dy;
      const float sv = acm_sample(src, sx + 0.5f, sy + 0.5f);
      if (rv > rc) rb |= 1u << bit;
      if (sv > sc) sb |= 1u << bit;
      ++bit;
    }
  const int ham = __popc(rb ^ sb);
  if (__popc(rb) < 3 && __popc(sb) < 3) return 1.0f;
  return (float)ham / 24.0f;
}

// The warp of the reference patch into one source (compute_cost_vector's
// per-view set-up, opencl_kernels.h:659-750): centre, the two affine steps
// and the source value at the centre.
struct SrcWarp {
  float scx, scy, ax, ay, bx, by, sc;
};

// single_cost's set-up of source i; false (cost 2) where a projection falls
// behind the source camera.
__device__ inline bool warp_setup(const AScene& S, int i, float3 cw, float3 wdx, float3 wdy,
                                  SrcWarp& w) {
  const ACam& c = S.cam[1 + i];
  const float3 p = acm_project(c, cw);
  if (p.z < 1e-6f) return false;
  w.scx = p.x / p.z;
  w.scy = p.y / p.z;
  const float3 pdx = acm_project(c, wdx), pdy = acm_project(c, wdy);
  if (pdx.z < 1e-6f || pdy.z < 1e-6f) return false;
  w.ax = pdx.x / pdx.z - w.scx;
  w.ay = pdx.y / pdx.z - w.scy;
  w.bx = pdy.x / pdy.z - w.scx;
  w.by = pdy.y / pdy.z - w.scy;
  w.sc = acm_sample(S.img[1 + i], w.scx + 0.5f, w.scy + 0.5f);
  return true;
}

// single_cost's tail from the multi-scale NCC of source i.
__device__ inline float finish_cost(const AScene& S, int i, const SrcWarp& w, float ncc, float rc,
                                    int cx, int cy) {
  const AImg& ref = S.img[0];
  const AImg& src = S.img[1 + i];
  if (ncc <= -0.5f) {
    if (S.census_weight > 1e-6f)
      return census(ref, src, rc, w.sc, cx, cy, w.scx, w.scy, w.ax, w.ay, w.bx, w.by);
    return 2.0f;
  }
  const float nc = 1.0f - ncc;
  if (S.census_weight < 1e-6f) return nc;
  const float t = acm_clamp((nc - 0.1f) / (0.6f - 0.1f), 0.0f, 1.0f);
  const float blend = S.census_weight * ((t * t) * (3.0f - 2.0f * t));
  if (blend < 1e-4f) return nc;
  const float cen = census(ref, src, rc, w.sc, cx, cy, w.scx, w.scy, w.ax, w.ay, w.bx, w.by);
  return (1.0f - blend) * nc + blend * cen;
}

// One source's cost: the warp set-up, the multi-scale NCC and the tail.
__device__ float single_cost(const AScene& S, int i, float3 cw, float3 wdx, float3 wdy, float rc,
                             int cx, int cy, float sf, float cf) {
  SrcWarp w;
  if (!warp_setup(S, i, cw, wdx, wdy, w)) return 2.0f;
  const float ncc = ncc_multiscale(S.img[0], S.img[1 + i], rc, w.sc, w.scx, w.scy, cx, cy,
                                   S.half_patch, w.ax, w.ay, w.bx, w.by, sf, cf);
  return finish_cost(S, i, w, ncc, rc, cx, cy);
}

// compute_cost_vector (opencl_kernels.h:659-750): out[0 .. n_src).
__device__ void cost_vector(const AScene& S, int x, int y, float4 plane, float* out) {
  const ACam& c0 = S.cam[0];
  const float depth = acm_depth(c0, (float)x, (float)y, plane);
  const float ddx = depth > 0.0f ? acm_depth(c0, (float)(x + 1), (float)y, plane) : 0.0f;
  const float ddy = depth > 0.0f ? acm_depth(c0, (float)x, (float)(y + 1), plane) : 0.0f;
  if (depth <= 0.0f || ddx <= 0.0f || ddy <= 0.0f) {
    for (int i = 0; i < S.n_src; ++i) out[i] = 2.0f;
    return;
  }
  const float3 cw = acm_backproject(c0, (float)x, (float)y, depth);
  const float3 wdx = acm_backproject(c0, (float)(x + 1), (float)y, ddx);
  const float3 wdy = acm_backproject(c0, (float)x, (float)(y + 1), ddy);
  const float rc = acm_texel(S.img[0], x, y);
  const float sf = -1.0f / (2.0f * S.sigma_spatial * S.sigma_spatial);
  const float cf = -1.0f / (2.0f * S.sigma_color * S.sigma_color);
  for (int i = 0; i < S.n_src; ++i) out[i] = single_cost(S, i, cw, wdx, wdy, rc, x, y, sf, cf);
}

__device__ float smoothness(const AScene& S, const float4* __restrict__ planes, float4 cur, int x,
                            int y) {
  const ACam& c = S.cam[0];
  const float cd = acm_depth(c, (float)x, (float)y, cur);
  if (cd <= 0.0f) return 0.0f;
  const float3 cn = acm_normalize(make_float3(cur.x, cur.y, cur.z));
  const float sig = 0.02f;
  float tw = 0.0f, tc = 0.0f;
  for (int k = 0; k < 4; ++k) {
    const int nx = x + (k == 0 ? -1 : (k == 1 ? 1 : 0));
    const int ny = y + (k == 2 ? -1 : (k == 3 ? 1 : 0));
    if (nx < 0 || nx >= S.W || ny < 0 || ny >= S.H) continue;
    const float4 nb = planes[(size_t)ny * S.W + nx];
    const float nd = acm_depth(c, (float)nx, (float)ny, nb);
    if (nd <= 0.0f) continue;
    const float rel = fabsf(cd - nd) / cd;
    const float w = acm_exp(-rel * rel / (2.0f * sig * sig));
    const float3 nn = acm_normalize(make_float3(nb.x, nb.y, nb.z));
    const float ncost = 1.0f - ((cn.x * nn.x + cn.y * nn.y) + cn.z * nn.z);
    const float pred = acm_depth(c, (float)nx, (float)ny, cur);
    const float dev = pred > 0.0f ? fabsf(nd - pred) / cd : 0.0f;
    const float cost =
        0.5f * acm_clamp(ncost, 0.0f, 1.0f) + 0.5f * acm_clamp(dev * 10.0f, 0.0f, 1.0f);
    tc += w * cost;
    tw += w;
  }
  if (tw < 1e-6f) return 0.0f;
  return tc / tw;
}

// compute_geom_consistency_cost (opencl_kernels.h:945-990): the forward-
// backward reprojection error through source i's previous-level depth
// (nearest pixel), at most 5 px.
__device__ float geom_cost(const AScene& S, int i, float4 plane, int px, int py) {
  const float maxc = 5.0f;
  const ACam& rc = S.cam[0];
  const ACam& sc = S.cam[1 + i];
  const float depth = acm_depth(rc, (float)px, (float)py, plane);
  if (depth <= 0.0f) return maxc;
  const float3 p = acm_project(sc, acm_backproject(rc, (float)px, (float)py, depth));
  if (p.z < 1e-6f) return maxc;
  const float sx = p.x / p.z, sy = p.y / p.z;
  if (sx < 0.0f || sx >= (float)S.W || sy < 0.0f || sy >= (float)S.H) return maxc;
  const int ix = clampi((int)(sx + 0.5f), S.W), iy = clampi((int)(sy + 0.5f), S.H);
  const float sd = S.prev[(size_t)i * S.W * S.H + (size_t)iy * S.W + ix];
  if (sd <= 0.0f) return maxc;
  const float3 rp = acm_project(rc, acm_backproject(sc, sx, sy, sd));
  if (rp.z < 1e-6f) return maxc;
  const float dx = (float)px - rp.x / rp.z, dy = (float)py - rp.y / rp.z;
  const float e = sqrtf(dx * dx + dy * dy);
  return e < maxc ? e : maxc;
}

// compute_weighted_cost_geom (opencl_kernels.h:1017-1045).
__device__ inline float weighted(const AScene& S, const float* cv, const float* vw, float norm,
                                 float4 plane, int x, int y) {
  if (norm < 1e-6f) return 2.0f;
  float total = 0.0f;
  for (int i = 0; i < S.n_src; ++i)
    if (vw[i] > 0.0f) {
      float geom = 0.0f;
      if (S.geom_weight > 0.0f && (S.prev_mask & (1u << i))) geom = geom_cost(S, i, plane, x, y);
      total += vw[i] * (cv[i] + S.geom_weight * geom);
    }
  return total / norm;
}

// ---------------------------------------------------------------- kernels
// acmmp_random_init (opencl_kernels.h:1055-1124), one thread per pixel.
__global__ void acm_init_kernel(const AScene* __restrict__ Sp, AState st) {
  const AScene& S = *Sp;
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= S.W || y >= S.H) return;
  const int idx = y * S.W + x;
  uint2 s = make_uint2((unsigned)idx * 1099087573u + 2654435769u, (unsigned)idx * 2246822519u + 13u);
  const unsigned key = (unsigned)(idx + 7919);
  const float lmin = acm_log(S.depth_min > 1e-6f ? S.depth_min : 1e-6f);
  const float lmax = acm_log(S.depth_max > 1e-5f ? S.depth_max : 1e-5f);
  const float depth = acm_exp(lmin + acm_rand(s, key) * (lmax - lmin));
  float3 n;
  n.x = acm_rand(s, key + 3u) * 2.0f - 1.0f;
  n.y = acm_rand(s, key + 5u) * 2.0f - 1.0f;
  n.z = -1.0f;
  n = acm_normalize(n);
  const float4 pl = acm_plane(S.cam[0], (float)x, (float)y, depth, n);
  st.planes[idx] = pl;
  st.rs[idx] = s;
  // compute_initial_cost_and_views (752-829): mean of the top-k costs and
  // the views at or below the k-th.
  float cv[kMaxSrc], cc[kMaxSrc];
  for (int i = 0; i < kMaxSrc; ++i) cv[i] = cc[i] = 2.0f;
  cost_vector(S, x, y, pl, cv);
  int nv = 0;
  for (int i = 0; i < S.n_src; ++i) {
    cc[i] = cv[i];
    nv += cv[i] < 2.0f;
  }
  for (int i = 1; i < S.n_src; ++i) {
    const float tmp = cv[i];
    int j = i;
    for (; j >= 1 && tmp < cv[j - 1]; --j) cv[j] = cv[j - 1];
    cv[j] = tmp;
  }
  unsigned sel = 0;
  const int k = min(min(S.top_k, nv), S.n_src);
  float cost = 2.0f;
  if (k > 0) {
    float total = 0.0f;
    for (int i = 0; i < k; ++i) total += cv[i];
    const float thr = cv[k - 1];
    for (int i = 0; i < S.n_src; ++i)
      if (cc[i] <= thr) sel |= 1u << i;
    cost = total / (float)k;
  }
  st.costs[idx] = cost;
  st.sel[idx] = sel;
}

// acmmp_upsample (opencl_kernels.h:1828-1892): each fine pixel takes its
// nearest coarse plane re-anchored at itself, or a random plane where the
// coarse depth is invalid; costs 2, views unselected, RNG states reset.
__global__ void acm_upsample_kernel(const AScene* __restrict__ Sp, AState st,
                                    const float4* __restrict__ src, int sw, int sh) {
  const AScene& S = *Sp;
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= S.W || y >= S.H) return;
  const int idx = y * S.W + x;
  uint2 s = make_uint2((unsigned)idx * 1099087573u + 2654435769u, (unsigned)idx * 2246822519u + 13u);
  const float scx = (float)sw / (float)S.W, scy = (float)sh / (float)S.H;
  const int sx = clampi((int)((float)x * scx), sw), sy = clampi((int)((float)y * scy), sh);
  const float4 pl = src[(size_t)sy * sw + sx];
  const ACam& c0 = S.cam[0];
  const float depth = acm_depth(c0, (float)x, (float)y, pl);
  if (depth > 0.0f) {
    st.planes[idx] = acm_plane(c0, (float)x, (float)y, depth, acm_normalize(make_float3(pl.x, pl.y, pl.z)));
  } else {
    const unsigned key = (unsigned)(idx + 7919);
    const float lmin = acm_log(S.depth_min > 1e-6f ? S.depth_min : 1e-6f);
    const float lmax = acm_log(S.depth_max > 1e-5f ? S.depth_max : 1e-5f);
    const float rd = acm_exp(lmin + acm_rand(s, key) * (lmax - lmin));
    float3 n;
    n.x = acm_rand(s, key + 3u) * 2.0f - 1.0f;
    n.y = acm_rand(s, key + 5u) * 2.0f - 1.0f;
    n.z = -1.0f;
    st.planes[idx] = acm_plane(c0, (float)x, (float)y, rd, acm_normalize(n));
  }
  st.rs[idx] = s;
  st.costs[idx] = 2.0f;
  st.sel[idx] = 0u;
}

// acmmp_patchmatch (opencl_kernels.h:1298-1826) for the pixels of one colour:
// x = 2 gx + ((y + colour) & 1).
// The NCC work queue of one warp in shared memory, for n sources: the
// lanes' pixels, the per-(lane, source) warps and NCC results, and the list
// of evaluations of the current stride.  96 + 272 n words.
__host__ __device__ constexpr int acm_queue_words(int n) { return 96 + 272 * n; }

struct WarpQueue {
  int* cx;
  int* cy;
  float* rc;
  SrcWarp* prm;          // [32][n]
  float* res;            // [32][n]
  unsigned short* list;  // [32 n]: lane << 4 | source
};

__device__ inline WarpQueue warp_queue(float* base, int n) {
  WarpQueue q;
  q.cx = reinterpret_cast<int*>(base);
  q.cy = reinterpret_cast<int*>(base + 32);
  q.rc = base + 64;
  q.prm = reinterpret_cast<SrcWarp*>(base + 96);
  q.res = base + 96 + 224 * n;
  q.list = reinterpret_cast<unsigned short*>(base + 96 + 256 * n);
  return q;
}

// cost_vector for the 32 pixels of a warp, called by all its lanes together
// (`act` false: the lane wants no costs and `out` is left alone).  Per
// stride, the NCC evaluations still needed, one per (pixel, source), are
// listed and spread over the lanes, so the warp walks each stride's patch
// once per 32 evaluations instead of once per source with the lanes that
// are done idle.  Each evaluation is the sequential walk of ncc_at_stride,
// and each pixel's strides are decided as in ncc_multiscale, so the costs
// are those of cost_vector.
__device__ void cost_vector_warp(const AScene& S, const WarpQueue& q, int lane, bool act, int x,
                                 int y, float4 plane, float* out) {
  const int n_src = S.n_src;
  unsigned on = 0u;
  float rc = 0.0f;
  if (act) {
    const ACam& c0 = S.cam[0];
    const float depth = acm_depth(c0, (float)x, (float)y, plane);
    const float ddx = depth > 0.0f ? acm_depth(c0, (float)(x + 1), (float)y, plane) : 0.0f;
    const float ddy = depth > 0.0f ? acm_depth(c0, (float)x, (float)(y + 1), plane) : 0.0f;
    if (depth > 0.0f && ddx > 0.0f && ddy > 0.0f) {
      const float3 cw = acm_backproject(c0, (float)x, (float)y, depth);
      const float3 wdx = acm_backproject(c0, (float)(x + 1), (float)y, ddx);
      const float3 wdy = acm_backproject(c0, (float)x, (float)(y + 1), ddy);
      rc = acm_texel(S.img[0], x, y);
      for (int i = 0; i < n_src; ++i) {
        SrcWarp w;
        if (warp_setup(S, i, cw, wdx, wdy, w)) {
          on |= 1u << i;
          q.prm[lane * n_src + i] = w;
        }
      }
    }
    for (int i = 0; i < n_src; ++i) out[i] = -1.0f;  // the best NCC so far
  }
  q.cx[lane] = x;
  q.cy[lane] = y;
  q.rc[lane] = rc;
  const float sf = -1.0f / (2.0f * S.sigma_spatial * S.sigma_spatial);
  const float cf = -1.0f / (2.0f * S.sigma_color * S.sigma_color);
  unsigned need = on, textureless = 0u;
  for (int st = 0; st < 3; ++st) {
    // Source-major order: consecutive lanes take neighbouring pixels of one
    // source, so their reads of that image stay close together.
    int total = 0;
    const unsigned below = (1u << lane) - 1u;
    for (int v = 0; v < n_src; ++v) {
      const bool mine = (need >> v) & 1u;
      const unsigned ball = __ballot_sync(0xffffffffu, mine);
      if (mine) q.list[total + __popc(ball & below)] = (unsigned short)((lane << 4) | v);
      total += __popc(ball);
    }
    if (total == 0) break;
    __syncwarp();
    const float stride = (float)(st + 1);
    for (int k = lane; k < total; k += 32) {
      const int item = q.list[k], l = item >> 4, v = item & 15;
      const SrcWarp w = q.prm[l * n_src + v];
      q.res[l * n_src + v] =
          ncc_at_stride(S.img[0], S.img[1 + v], q.rc[l], w.sc, w.scx, w.scy, q.cx[l], q.cy[l],
                        S.half_patch, stride, w.ax, w.ay, w.bx, w.by, sf, cf);
    }
    __syncwarp();
    for (unsigned m = need; m; m &= m - 1u) {
      const int i = __ffs((int)m) - 1;
      const unsigned bit = 1u << i;
      float n = q.res[lane * n_src + i];
      if (st == 0 && n < -0.5f) textureless |= bit;
      if ((textureless & bit) && n > 0.0f) n = 0.0f;
      if (n > out[i]) out[i] = n;
      if (out[i] > 0.1f) need &= ~bit;
    }
    __syncwarp();
  }
  if (act)
    for (int i = 0; i < n_src; ++i)
      out[i] = (on >> i) & 1u ? finish_cost(S, i, q.prm[lane * n_src + i], out[i], rc, x, y)
                              : 2.0f;
}

// acmmp_patchmatch (opencl_kernels.h:1298-1826) for one colour, one thread
// per pixel.  The 14 cost vectors of a pixel (8 propagation candidates, the
// current plane, 5 refinement hypotheses) are computed in that order by one
// call site, cost_vector_warp, which the whole warp enters together.  Eight
// blocks of two warps per SM (128 registers).
__global__ void __launch_bounds__(64, 8) acm_pm_kernel(const AScene* __restrict__ Sp, AState st,
                                                       int colour, int iteration) {
  extern __shared__ float acm_smem[];
  const AScene& S = *Sp;
  const int W = S.W, H = S.H, npix = W * H;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x, lane = tid & 31;
  const WarpQueue q = warp_queue(acm_smem + (tid >> 5) * acm_queue_words(S.n_src), S.n_src);
  int y = blockIdx.y * blockDim.y + threadIdx.y;
  int x = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((y + colour) & 1);
  // A lane outside the image stays with its warp on pixel (0, 0), asks for
  // no costs and writes nothing.
  const bool valid = x < W && y < H;
  if (!valid) x = y = 0;
  const int idx = y * W + x;
  const ACam& c0 = S.cam[0];
  uint2 s = st.rs[idx];
  const unsigned key = (unsigned)(idx + iteration * 7919 + 42);
  const int n_src = S.n_src;
  const float* C = st.costs;
  int pos[8];
  bool flags[8];
  float ca[8 * kMaxSrc];
  for (int i = 0; i < 8; ++i) {
    pos[i] = idx;
    flags[i] = false;
  }
  for (int i = 0; i < 8 * kMaxSrc; ++i) ca[i] = 2.0f;
  float vw[kMaxSrc];
  float norm = 0.0f;
  unsigned new_sel = 0;
  int best = 0;
  float bcost = 0.0f;
  float4 plane_now = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float cost_now = 0.0f, depth_now = 0.0f, depth_rand = 0.0f, depth_pert = 0.0f,
        depth_cur = 0.0f;
  float3 cur_n = make_float3(0.0f, 0.0f, -1.0f), nr = cur_n, np_ = cur_n;
  float cvh[kMaxSrc];
  for (int h = 0; h < 14; ++h) {
    bool act = valid;
    float4 pl = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float* outp = cvh;
    if (h < 8) {
      // Candidate positions in the reference's evaluation order: far up,
      // down, left, right (slots 1, 3, 5, 7), then near up, down, left,
      // right (0, 2, 4, 6).  Each slot takes the lowest-cost pixel of its
      // pattern.
      const int slot_i = h;
      bool found = false;
      do {
        const int slot = slot_i < 4 ? 2 * slot_i + 1 : 2 * (slot_i - 4);
        const int dir = slot >> 1;  // 0 up, 1 down, 2 left, 3 right
        const bool vert = dir < 2;
        const int sgn = (dir & 1) ? 1 : -1;
        int base;
        float bc;
        int bp;
        if (slot & 1) {  // far
          const bool ok =
              dir == 0 ? y > 2 : (dir == 1 ? y < H - 3 : (dir == 2 ? x > 2 : x < W - 3));
          if (!ok) break;
          base = vert ? (y + 3 * sgn) * W + x : y * W + (x + 3 * sgn);
          bc = C[base];
          bp = base;
          for (int i = 1; i < 11; ++i) {
            const int qc = vert ? y + sgn * (3 + 2 * i) : x + sgn * (3 + 2 * i);
            if (qc < 0 || qc >= (vert ? H : W)) break;
            const int pp = vert ? qc * W + x : y * W + qc;
            if (C[pp] < bc) {
              bc = C[pp];
              bp = pp;
            }
          }
        } else {  // near, with a V of diagonals behind the neighbour
          const bool ok =
              dir == 0 ? y > 0 : (dir == 1 ? y < H - 1 : (dir == 2 ? x > 0 : x < W - 1));
          if (!ok) break;
          base = vert ? (y + sgn) * W + x : y * W + (x + sgn);
          bc = C[base];
          bp = base;
          for (int i = 0; i < 3; ++i) {
            for (int side = 0; side < 2; ++side) {
              bool cond;
              int pp;
              if (vert) {
                const bool along = dir == 0 ? y > 1 + i : y < H - 2 - i;
                cond = along && (side == 0 ? x > i : x < W - 1 - i);
                pp = (y + sgn * (2 + i)) * W + (side == 0 ? x - i - 1 : x + i + 1);
              } else {
                const bool along = dir == 2 ? x > 1 + i : x < W - 2 - i;
                cond = along && (side == 0 ? y > i : y < H - 1 - i);
                pp = (side == 0 ? y - i - 1 : y + i + 1) * W + (x + sgn * (2 + i));
              }
              if (cond && pp >= 0 && pp < npix && C[pp] < bc) {
                bc = C[pp];
                bp = pp;
              }
            }
          }
        }
        pos[slot] = bp;
        flags[slot] = true;
        pl = st.planes[bp];
        outp = &ca[slot * kMaxSrc];
        found = true;
      } while (false);
      act = act && found;
    } else {
      for (int i = 0; i < kMaxSrc; ++i) cvh[i] = 2.0f;
      if (h == 8) {
        pl = st.planes[idx];
      } else {
        const int r = h - 9;
        const float dh = r == 0 || r == 2 ? depth_rand : (r == 4 ? depth_pert : depth_cur);
        const float3 nh = r == 1 || r == 2 ? nr : (r == 3 ? np_ : cur_n);
        pl = acm_plane(c0, (float)x, (float)y, dh, nh);
      }
    }
    cost_vector_warp(S, q, lane, act, x, y, pl, outp);
    if (h == 7) {
      // View selection priors from the four direct neighbours (last one wins).
      float pri[kMaxSrc];
      for (int i = 0; i < kMaxSrc; ++i) pri[i] = 0.0f;
      const int npos[4] = {idx - W, idx + W, idx - 1, idx + 1};
      for (int i = 0; i < 4; ++i) {
        const int np = npos[i];
        if (flags[2 * i] && np >= 0 && np < npix) {
          const unsigned sv = st.sel[np];
          for (int j = 0; j < n_src; ++j) pri[j] = (sv & (1u << j)) ? 0.9f : 0.1f;
        }
      }
      const float thr = 0.8f * acm_exp((float)(iteration * iteration) / (-90.0f));
      float prob[kMaxSrc];
      for (int i = 0; i < kMaxSrc; ++i) prob[i] = 0.0f;
      for (int i = 0; i < n_src; ++i) {
        float count = 0.0f, tw = 0.0f;
        int cfalse = 0;
        for (int j = 0; j < 8; ++j) {
          const float cv = ca[j * kMaxSrc + i];
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
      {
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
      for (int i = 0; i < kMaxSrc; ++i) vw[i] = 0.0f;
      for (int smp = 0; smp < 15; ++smp) {
        const float r = acm_rand(s, key + (unsigned)smp * 997u) - 1e-7f;
        for (int j = 0; j < n_src; ++j)
          if (prob[j] > r) {
            vw[j] += 1.0f;
            break;
          }
      }
      for (int i = 0; i < n_src; ++i)
        if (vw[i] > 0.0f) {
          new_sel |= 1u << i;
          norm += vw[i];
        }
      for (int i = 0; i < 8; ++i) {
        float fc = 2.0f;
        if (flags[i]) {
          const float photo =
              weighted(S, &ca[i * kMaxSrc], vw, norm, st.planes[pos[i]], x, y);
          fc = S.smooth_weight > 1e-6f
                   ? photo + S.smooth_weight * smoothness(S, st.planes, st.planes[pos[i]], x, y)
                   : photo;
        }
        if (i == 0 || fc < bcost) {
          bcost = fc;
          best = i;
        }
      }
    } else if (h == 8) {
      const float4 own = pl;
      cost_now = weighted(S, cvh, vw, norm, own, x, y);
      if (S.smooth_weight > 1e-6f)
        cost_now += S.smooth_weight * smoothness(S, st.planes, own, x, y);
      plane_now = own;
      depth_now = acm_depth(c0, (float)x, (float)y, plane_now);
      if (flags[best] && bcost < cost_now) {
        const float4 bpl = st.planes[pos[best]];
        const float db = acm_depth(c0, (float)x, (float)y, bpl);
        if (db >= S.depth_min && db <= S.depth_max) {
          depth_now = db;
          plane_now = bpl;
          cost_now = bcost;
          if (valid) st.sel[idx] = new_sel;
        }
      }
      // Refinement: (random depth, current normal), (current depth, random
      // normal), (random, random), (current, perturbed normal), (perturbed
      // depth, current normal).
      const float pert = 0.02f;
      const float PI_F = 3.14159274101257324f;
      cur_n = acm_normalize(make_float3(plane_now.x, plane_now.y, plane_now.z));
      // The SfM planar prior (where it covers the pixel) centres the random
      // hypothesis on its plane: depth within 3 sigma, normal within 5
      // degrees.
      const bool have_prior = S.prior_mask != nullptr && S.prior_mask[idx] > 0u;
      float depth_prior = 0.0f;
      float3 prior_n = make_float3(0.0f, 0.0f, -1.0f);
      if (have_prior) {
        const float4 pp = S.prior_planes[idx];
        depth_prior = acm_depth(c0, (float)x, (float)y, pp);
        prior_n = acm_normalize(make_float3(pp.x, pp.y, pp.z));
      }
      if (have_prior && depth_prior > 0.0f) {
        const float depth_sigma = (S.depth_max - S.depth_min) / 32.0f;
        const float angle_sigma = PI_F * (5.0f / 180.0f);
        depth_rand =
            depth_prior - 3.0f * depth_sigma + acm_rand(s, key + 503u) * 6.0f * depth_sigma;
        depth_rand = acm_clamp(depth_rand, S.depth_min, S.depth_max);
        const float q1 = (acm_rand(s, key + 504u) - 0.5f) * angle_sigma;
        const float q2 = (acm_rand(s, key + 505u) - 0.5f) * angle_sigma;
        nr = acm_normalize(make_float3(prior_n.x + q1, prior_n.y + q2, prior_n.z));
        if (nr.z > 0.0f) nr.z = -nr.z;
      } else {
        const float lmin = acm_log(S.depth_min > 1e-6f ? S.depth_min : 1e-6f);
        const float lmax = acm_log(S.depth_max > 1e-5f ? S.depth_max : 1e-5f);
        depth_rand = acm_exp(lmin + acm_rand(s, key + 503u) * (lmax - lmin));
        nr.x = acm_rand(s, key + 504u) * 2.0f - 1.0f;
        nr.y = acm_rand(s, key + 505u) * 2.0f - 1.0f;
        nr.z = -1.0f;
        nr = acm_normalize(nr);
      }
      const float dmn = (1.0f - pert) * depth_now, dmx = (1.0f + pert) * depth_now;
      depth_pert =
          acm_clamp(dmn + acm_rand(s, key + 510u) * (dmx - dmn), S.depth_min, S.depth_max);
      const float pa1 = ((acm_rand(s, key + 520u) - 0.5f) * pert) * PI_F;
      const float pa2 = ((acm_rand(s, key + 521u) - 0.5f) * pert) * PI_F;
      np_ = acm_normalize(make_float3(cur_n.x + pa1, cur_n.y + pa2, cur_n.z));
      if (np_.z > 0.0f) np_.z = -np_.z;
      depth_cur = depth_now;  // the five hypotheses are fixed before any is taken
    } else if (h > 8) {
      const float4 cand = pl;
      float tc = weighted(S, cvh, vw, norm, cand, x, y);
      if (S.smooth_weight > 1e-6f) tc += S.smooth_weight * smoothness(S, st.planes, cand, x, y);
      const float db = acm_depth(c0, (float)x, (float)y, cand);
      if (!(db < S.depth_min || db > S.depth_max) && tc < cost_now) {
        depth_now = db;
        plane_now = cand;
        cost_now = tc;
      }
    }
  }
  if (valid) {
    st.planes[idx] = plane_now;
    st.costs[idx] = cost_now;
    st.rs[idx] = s;
  }
}

// acmmp_checkerboard_filter (opencl_kernels.h:1919-2099) for one colour.
__global__ void acm_filter_kernel(const AScene* __restrict__ Sp, AState st, int colour) {
  const AScene& S = *Sp;
  const int W = S.W, H = S.H;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + ((y + colour) & 1);
  if (x >= W || y >= H) return;
  const int c = y * W + x;
  if (st.costs[c] < 0.001f) return;
  const ACam& c0 = S.cam[0];
  // The 20 neighbours in the reference's order: (dx, dy) and their bounds.
  const int ox[20] = {0, 0, 0, 0, 0, 0, -1, -3, -5, 1, 3, 5, 2, 2, -2, -2, -1, 1, -1, 1};
  const int oy[20] = {-1, -3, -5, 1, 3, 5, 0, 0, 0, 0, 0, 0, -1, 1, -1, 1, -2, -2, 2, 2};
  float buf[21];
  int n = 0;
  buf[n++] = acm_depth(c0, (float)x, (float)y, st.planes[c]);
  for (int k = 0; k < 20; ++k) {
    const int dx = ox[k], dy = oy[k];
    bool ok;
    if (k < 6)
      ok = dy < 0 ? y > -dy - 1 : y < H - dy;
    else if (k < 12)
      ok = dx < 0 ? x > -dx - 1 : x < W - dx;
    else if (k < 16)
      ok = (dy < 0 ? y > 0 : y < H - 1) && (dx > 0 ? x < W - 2 : x > 1);
    else
      ok = (dx < 0 ? x > 0 : x < W - 1) && (dy < 0 ? y > 2 : y < H - 2);
    if (ok) buf[n++] = acm_depth(c0, (float)(x + dx), (float)(y + dy), st.planes[c + dy * W + dx]);
  }
  const float cd = buf[0];
  if (cd > 0.0f) {
    const float lo = cd * (1 - 0.15f), hi = cd * (1 + 0.15f);
    int m = 1;
    for (int i = 1; i < n; ++i)
      if (buf[i] > lo && buf[i] < hi) buf[m++] = buf[i];
    n = m;
  }
  for (int i = 1; i < n; ++i) {
    const float t = buf[i];
    int j = i;
    for (; j >= 1 && t < buf[j - 1]; --j) buf[j] = buf[j - 1];
    buf[j] = t;
  }
  const int mid = n / 2;
  const float med = (n % 2 == 0) ? (buf[mid - 1] + buf[mid]) * 0.5f : buf[mid];
  if (med > 0.0f) {
    const float4 p = st.planes[c];
    st.planes[c] = acm_plane(c0, (float)x, (float)y, med, acm_normalize(make_float3(p.x, p.y, p.z)));
  }
}

// ReadBackResults (estimator.cc:958-1000): depth, unit normal, cost.
__global__ void acm_readback_kernel(const AScene* __restrict__ Sp, AState st,
                                    float* __restrict__ depth, float* __restrict__ normal,
                                    float* __restrict__ cost) {
  const AScene& S = *Sp;
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= S.W || y >= S.H) return;
  const size_t i = (size_t)y * S.W + x;
  const float4 p = st.planes[i];
  float d = 0.0f, n0 = 0.0f, n1 = 0.0f, n2 = 0.0f, cs = 0.0f;
  if (isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(p.w)) {
    const ACam& c = S.cam[0];
    const float r0 = ((float)x - c.K[2]) / c.K[0], r1 = ((float)y - c.K[5]) / c.K[4];
    const float den = (p.x * r0 + p.y * r1) + p.z * 1.0f;
    float dd = fabsf(den) > 1e-6f ? -p.w / den : 0.0f;
    if (!isfinite(dd)) dd = 0.0f;
    if (dd > 0.0f && dd >= S.depth_min && dd <= S.depth_max) {
      d = dd;
      const float len = sqrtf((p.x * p.x + p.y * p.y) + p.z * p.z);
      if (len > 1e-6f) {
        n0 = p.x / len;
        n1 = p.y / len;
        n2 = p.z / len;
      }
    }
    const float cc = st.costs[i];
    cs = isfinite(cc) ? cc : 0.0f;
  }
  depth[i] = d;
  normal[3 * i] = n0;
  normal[3 * i + 1] = n1;
  normal[3 * i + 2] = n2;
  cost[i] = cs;
}

// The 5x5 median rejection (estimator.cc:1004-1021, cv::medianBlur with
// replicated borders): depth d is zeroed where the median m > 0 and
// |d - m| / d > 0.10.
__global__ void acm_median_kernel(int W, int H, const float* __restrict__ depth,
                                  float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  float v[25];
  int k = 0;
  for (int a = -2; a <= 2; ++a)
    for (int b = -2; b <= 2; ++b) v[k++] = depth[(size_t)clampi(y + a, H) * W + clampi(x + b, W)];
  for (int i = 1; i < 25; ++i) {
    const float t = v[i];
    int j = i;
    for (; j >= 1 && t < v[j - 1]; --j) v[j] = v[j - 1];
    v[j] = t;
  }
  const float d = depth[(size_t)y * W + x], m = v[12];
  out[(size_t)y * W + x] = (d > 0.0f && m > 0.0f && fabsf(d - m) / d > 0.10f) ? 0.0f : d;
}

// ------------------------------------------------------------------ host
// The stream a level runs on, for stream-ordered allocation: references run
// concurrently on their own streams, and a plain cudaFree would wait for the
// whole device.
thread_local cudaStream_t tl_stream = nullptr;

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, tl_stream);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    if (count <= n && p) return cudaSuccess;
    release();
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&p),
                                    std::max<size_t>(count, 1) * sizeof(T), tl_stream);
    if (e == cudaSuccess) n = count;
    return e;
  }
};

struct AView {
  double K[9], R[9], t[3];
  int W, H;
  std::vector<uint8_t> img;
};
struct ARef {
  std::vector<AView> views;  // [0] the reference
  float depth_min, depth_max;
  std::vector<double> sfm;  // SfM points (world, rows of 3) for the planar prior
  int W = 0, H = 0;  // size of the result
  std::vector<float> depth, normal, cost, conf;
};

}  // namespace

struct dn_acmmp {
  int device = 0;
  cudaStream_t stream = nullptr;
  // DepthmapParams defaults (estimator.h:17-31).
  int max_iterations = 3, patch_size = 11, max_image_size = 3200, hierarchy_levels = 1;
  float sigma_spatial = 5.0f, sigma_color = 3.0f / 255.0f;
  int top_k = 4;
  float census_weight = 0.3f, smooth_weight = 0.0f, geom_weight = 0.0f;
  std::vector<ARef> refs;
  std::vector<int> geom_links;  // (ref, source, from) triples
  float last_ms = 0.0f;
  ~dn_acmmp() {
    if (stream) cudaStreamDestroy(stream);
  }
};

extern "C" const char* dn_acmmp_last_error(void) { return g_acm_error.c_str(); }



extern "C" dn_status dn_acmmp_create(dn_acmmp** out) {
  const dn::DeviceRestore device_restore_;
  ACHECK(out, "NULL output");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return afail(DN_DEVICE_ERROR, "no CUDA device");
  auto e = std::make_unique<dn_acmmp>();
  ACUDA(cudaGetDevice(&e->device));
  ACUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  *out = e.release();
  return DN_OK;
}
extern "C" dn_status dn_acmmp_destroy(dn_acmmp* e) {
  const dn::DeviceRestore device_restore_;
  delete e;
  return DN_OK;
}

#define ACM_SETTER(name, field, type)                           \
  extern "C" dn_status dn_acmmp_set_##name(dn_acmmp* e, type v) { \
    ACHECK(e, "NULL estimator");                                \
    e->field = v;                                               \
    return DN_OK;                                               \
  }
ACM_SETTER(max_iterations, max_iterations, int)
ACM_SETTER(max_image_size, max_image_size, int)
ACM_SETTER(hierarchy_levels, hierarchy_levels, int)
ACM_SETTER(sigma_spatial, sigma_spatial, float)
ACM_SETTER(sigma_color, sigma_color, float)
ACM_SETTER(top_k, top_k, int)
ACM_SETTER(census_weight, census_weight, float)
ACM_SETTER(smooth_weight, smooth_weight, float)
ACM_SETTER(geom_consistency_weight, geom_weight, float)
#undef ACM_SETTER

extern "C" dn_status dn_acmmp_set_patch_size(dn_acmmp* e, int size) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e, "NULL estimator");
  ACHECK(size >= 1 && size <= 63, "patch size must be in [1, 63]");
  e->patch_size = size;
  return DN_OK;
}

extern "C" dn_status dn_acmmp_set_device(dn_acmmp* e, int device) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e, "NULL estimator");
  int n = 0;
  ACUDA(cudaGetDeviceCount(&n));
  ACHECK(device >= 0 && device < n, "no such CUDA device");
  ACUDA(cudaSetDevice(device));
  cudaStream_t s;
  ACUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  cudaSetDevice(e->device);
  cudaStreamDestroy(e->stream);
  e->stream = s;
  e->device = device;
  return DN_OK;
}

static dn_status make_view(const double* K, const double* R, const double* t,
                           const uint8_t* img, int w, int h, int stride, AView* v) {
  ACHECK(K && R && t && img, "NULL argument");
  ACHECK(w >= 1 && h >= 1 && w <= 16384 && h <= 16384, "bad image size");
  ACHECK(stride >= w, "stride below width");
  for (int i = 0; i < 9; ++i) ACHECK(std::isfinite(K[i]) && std::isfinite(R[i]), "K, R must be finite");
  for (int i = 0; i < 3; ++i) ACHECK(std::isfinite(t[i]), "t must be finite");
  std::memcpy(v->K, K, sizeof(v->K));
  std::memcpy(v->R, R, sizeof(v->R));
  std::memcpy(v->t, t, sizeof(v->t));
  v->W = w;
  v->H = h;
  v->img.resize((size_t)w * h);
  for (int r = 0; r < h; ++r) std::memcpy(&v->img[(size_t)r * w], img + (size_t)r * stride, w);
  return DN_OK;
}

extern "C" dn_status dn_acmmp_begin_ref_view(dn_acmmp* e, const double* K, const double* R,
                                             const double* t, const uint8_t* img, int w, int h,
                                             int stride, float depth_min, float depth_max,
                                             int* ref_idx) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e, "NULL estimator");
  ARef ref;
  ref.depth_min = depth_min;
  ref.depth_max = depth_max;
  ref.views.emplace_back();
  const dn_status st = make_view(K, R, t, img, w, h, stride, &ref.views.back());
  if (st != DN_OK) return st;
  e->refs.push_back(std::move(ref));
  if (ref_idx) *ref_idx = (int)e->refs.size() - 1;
  return DN_OK;
}

extern "C" dn_status dn_acmmp_add_source_view(dn_acmmp* e, const double* K, const double* R,
                                              const double* t, const uint8_t* img, int w, int h,
                                              int stride) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e, "NULL estimator");
  if (e->refs.empty()) return afail(DN_INVALID_ARG, "DepthmapClusterEstimator: no ref view started");
  AView v;
  const dn_status st = make_view(K, R, t, img, w, h, stride, &v);
  if (st != DN_OK) return st;
  e->refs.back().views.push_back(std::move(v));
  return DN_OK;
}

extern "C" dn_status dn_acmmp_set_sfm_points(dn_acmmp* e, const double* points, int64_t n) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e, "NULL estimator");
  if (e->refs.empty()) return afail(DN_INVALID_ARG, "DepthmapClusterEstimator: no ref view started");
  ACHECK(n >= 0 && (n == 0 || points), "NULL points");
  for (int64_t i = 0; i < 3 * n; ++i) ACHECK(std::isfinite(points[i]), "SfM points must be finite");
  // SetSfMPoints (estimator.cc:108-118) replaces the reference's points.
  e->refs.back().sfm.assign(points, points + 3 * n);
  return DN_OK;
}

extern "C" dn_status dn_acmmp_add_geom_link(dn_acmmp* e, int ref_idx, int source_view_idx,
                                            int from_ref_idx) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e, "NULL estimator");
  ACHECK(ref_idx >= 0 && ref_idx < (int)e->refs.size(),
         "DepthmapClusterEstimator::AddGeomLink: invalid ref_idx");
  // Used only between pyramid levels (cluster_estimator.cc:107-125); with
  // one level the link has no effect, as in the reference.
  e->geom_links.insert(e->geom_links.end(), {ref_idx, source_view_idx, from_ref_idx});
  return DN_OK;
}

extern "C" dn_status dn_acmmp_clear(dn_acmmp* e) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e, "NULL estimator");
  e->refs.clear();
  e->geom_links.clear();
  return DN_OK;
}

extern "C" dn_status dn_acmmp_num_refs(dn_acmmp* e, int* n) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e && n, "NULL argument");
  *n = (int)e->refs.size();
  return DN_OK;
}

// cv::resize(INTER_AREA) of an 8-bit image by an integer factor k that
// divides both sizes (OpenCV's fast area path): the k x k block mean, rounded
// half up for k = 2, else float(sum) * float(1/k^2) rounded to nearest even.
static void resize_area_u8(const uint8_t* src, int W, int H, int k, uint8_t* dst) {
  const int w = W / k, h = H / k;
  const float inv = 1.0f / (float)(k * k);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      int sum = 0;
      for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) sum += src[(size_t)(k * y + a) * W + (k * x + b)];
      const int v = k == 2 ? (sum + 2) >> 2 : (int)std::nearbyint((float)sum * inv);
      dst[(size_t)y * w + x] = (uint8_t)std::min(255, std::max(0, v));
    }
}

// cv::resize(INTER_AREA) of an 8-bit image to (w, h) when the ratios are not
// both integers (OpenCV's general area path): per axis a table of source
// cells and float weights (overlap over cell width), a horizontal pass per
// source row and a vertical accumulation in float, rounded half to even.
struct AreaTab {
  int di, si;
  float alpha;
};

static int area_table(int ssize, int dsize, double scale, AreaTab* t) {
  int k = 0;
  for (int dx = 0; dx < dsize; ++dx) {
    const double fsx1 = dx * scale, fsx2 = fsx1 + scale;
    const double cell = std::min(scale, ssize - fsx1);
    int sx1 = (int)std::ceil(fsx1), sx2 = (int)std::floor(fsx2);
    sx2 = std::min(sx2, ssize - 1);
    sx1 = std::min(sx1, sx2);
    if (sx1 - fsx1 > 1e-3) t[k++] = AreaTab{dx, sx1 - 1, (float)((sx1 - fsx1) / cell)};
    for (int sx = sx1; sx < sx2; ++sx) t[k++] = AreaTab{dx, sx, (float)(1.0 / cell)};
    if (fsx2 - sx2 > 1e-3)
      t[k++] = AreaTab{dx, sx2, (float)(std::min(std::min(fsx2 - sx2, 1.0), cell) / cell)};
  }
  return k;
}

static void resize_area_general_u8(const uint8_t* src, int W, int H, uint8_t* dst, int w, int h) {
  const double sx = 1.0 / ((double)w / W), sy = 1.0 / ((double)h / H);
  std::vector<AreaTab> xt(2 * (size_t)(W + 2)), yt(2 * (size_t)(H + 2));
  std::vector<float> buf(w), sum(w);
  const int nx = area_table(W, w, sx, xt.data()), ny = area_table(H, h, sy, yt.data());
  auto flush = [&](int row) {
    for (int dx = 0; dx < w; ++dx) {
      const int v = (int)std::nearbyint(sum[dx]);
      dst[(size_t)row * w + dx] = (uint8_t)std::min(255, std::max(0, v));
    }
  };
  int prev = -1;
  for (int j = 0; j < ny; ++j) {
    const int dy = yt[j].di;
    const float beta = yt[j].alpha;
    const uint8_t* S = src + (size_t)yt[j].si * W;
    std::fill(buf.begin(), buf.end(), 0.0f);
    for (int k = 0; k < nx; ++k) buf[xt[k].di] += (float)S[xt[k].si] * xt[k].alpha;
    if (dy != prev) {
      if (prev >= 0) flush(prev);
      for (int dx = 0; dx < w; ++dx) sum[dx] = beta * buf[dx];
      prev = dy;
    } else {
      for (int dx = 0; dx < w; ++dx) sum[dx] += beta * buf[dx];
    }
  }
  if (prev >= 0) flush(prev);
}

// The previous-level depth resize (UploadPreviousDepths uses INTER_LINEAR):
// OpenCV's pixel-centre mapping, FP32 weights, each operation rounded by
// itself.  OpenCV's SIMD arithmetic can differ from this in the last bits.
static void resize_linear_f32(const float* src, int w, int h, float* dst, int W, int H) {
  for (int y = 0; y < H; ++y) {
    const double fyd = (y + 0.5) * ((double)h / H) - 0.5;
    int sy = (int)std::floor(fyd);
    float fy = (float)(fyd - sy);
    if (sy < 0) {
      sy = 0;
      fy = 0.0f;
    }
    if (sy >= h - 1) {
      sy = h - 1;
      fy = 0.0f;
    }
    const int sy1 = std::min(sy + 1, h - 1);
    for (int x = 0; x < W; ++x) {
      const double fxd = (x + 0.5) * ((double)w / W) - 0.5;
      int sx = (int)std::floor(fxd);
      float fx = (float)(fxd - sx);
      if (sx < 0) {
        sx = 0;
        fx = 0.0f;
      }
      if (sx >= w - 1) {
        sx = w - 1;
        fx = 0.0f;
      }
      const int sx1 = std::min(sx + 1, w - 1);
      const float a0 = 1.0f - fx, b0 = 1.0f - fy;
      const float r0 = src[(size_t)sy * w + sx] * a0 + src[(size_t)sy * w + sx1] * fx;
      const float r1 = src[(size_t)sy1 * w + sx] * a0 + src[(size_t)sy1 * w + sx1] * fx;
      dst[(size_t)y * W + x] = r0 * b0 + r1 * fy;
    }
  }
}

// Delaunay triangulation of 2-D points inside the image rectangle
// [0, w) x [0, h) (Bowyer-Watson, double precision).  The reference builds
// it with cv::Subdiv2D, which starts from the virtual triangle (3M, 0),
// (0, 3M), (-3M, -3M), M = max(w, h), and drops the triangles that touch
// it; so does this, and the result is the Delaunay triangulation of the
// points with those three vertices, less theirs.  Exact duplicates join the
// first.  Returns triangles as ascending index triples, sorted.
struct Tri {
  int a, b, c;
};

static std::vector<Tri> delaunay(const std::vector<double>& px, const std::vector<double>& py,
                                 int w, int h) {
  const int n = (int)px.size();
  std::vector<Tri> out;
  if (n < 3) return out;
  const double big = 3.0 * (double)std::max(w, h);
  std::vector<double> X(px), Y(py);
  X.push_back(big);
  Y.push_back(0.0);
  X.push_back(0.0);
  Y.push_back(big);
  X.push_back(-big);
  Y.push_back(-big);
  // Counter-clockwise triangles; nb[k] is the triangle across the edge
  // opposite v[k] (-1 on the outer triangle's edges).
  struct T {
    int v[3], nb[3];
    double cx, cy, r2;
    bool alive;
  };
  std::vector<T> tris;
  tris.reserve(8 * (size_t)n + 16);
  auto make = [&](int a, int b, int c) {
    T t;
    t.v[0] = a;
    t.v[1] = b;
    t.v[2] = c;
    t.nb[0] = t.nb[1] = t.nb[2] = -1;
    t.alive = true;
    const double ax = X[a], ay = Y[a], bx = X[b], by = Y[b], cx = X[c], cy = Y[c];
    const double d = 2.0 * (ax * (by - cy) + bx * (cy - ay) + cx * (ay - by));
    if (d == 0.0) {
      t.cx = t.cy = 0.0;
      t.r2 = -1.0;  // degenerate: its circle contains no point
    } else {
      const double a2 = ax * ax + ay * ay, b2 = bx * bx + by * by, c2 = cx * cx + cy * cy;
      t.cx = (a2 * (by - cy) + b2 * (cy - ay) + c2 * (ay - by)) / d;
      t.cy = (a2 * (cx - bx) + b2 * (ax - cx) + c2 * (bx - ax)) / d;
      t.r2 = (ax - t.cx) * (ax - t.cx) + (ay - t.cy) * (ay - t.cy);
    }
    tris.push_back(t);
    return (int)tris.size() - 1;
  };
  // The strict circumcircle test of Bowyer-Watson.
  auto bad = [&](const T& t, int i) {
    const double dx = X[i] - t.cx, dy = Y[i] - t.cy;
    return t.alive && t.r2 >= 0.0 && dx * dx + dy * dy < t.r2;
  };
  auto orient = [&](int a, int b, int i) {  // > 0: i left of a -> b
    return (X[b] - X[a]) * (Y[i] - Y[a]) - (Y[b] - Y[a]) * (X[i] - X[a]);
  };
  make(n, n + 1, n + 2);
  std::map<std::pair<double, double>, int> seen;  // distinct positions
  std::vector<int> mark;  // mark[u] == i: triangle u is in point i's cavity
  std::vector<int> cavity, stack, first_of(n + 3, -1), last_of(n + 3, -1), fresh;
  int last = 0;
  for (int i = 0; i < n; ++i) {
    if (!std::isfinite(X[i]) || !std::isfinite(Y[i])) continue;
    if (!seen.emplace(std::make_pair(X[i], Y[i]), i).second) continue;  // a duplicate
    // Locate: walk from the last new triangle towards the point.
    int t = last, steps = 0;
    const int max_steps = 4 * (int)tris.size() + 16;
    while (t >= 0 && steps++ < max_steps) {
      const T& c = tris[t];
      int next = -2;
      for (int k = 0; k < 3; ++k)
        if (orient(c.v[(k + 1) % 3], c.v[(k + 2) % 3], i) < 0.0) {
          next = c.nb[k];
          break;
        }
      if (next == -2) break;  // inside (or on an edge of) t
      t = next;
    }
    // The cavity: the triangles whose circles contain the point, grown
    // across neighbours from the located one; a full scan where the walk
    // or the located triangle's test fails numerically.
    mark.resize(tris.size(), -1);
    cavity.clear();
    if (t >= 0 && steps <= max_steps && bad(tris[t], i)) {
      stack.assign(1, t);
      mark[t] = i;
      while (!stack.empty()) {
        const int u = stack.back();
        stack.pop_back();
        cavity.push_back(u);
        for (int k = 0; k < 3; ++k) {
          const int v = tris[u].nb[k];
          if (v >= 0 && mark[v] != i && bad(tris[v], i)) {
            mark[v] = i;
            stack.push_back(v);
          }
        }
      }
    } else {
      for (int u = 0; u < (int)tris.size(); ++u)
        if (bad(tris[u], i)) {
          mark[u] = i;
          cavity.push_back(u);
        }
    }
    // A fan from the point over the cavity's boundary edges, linked to the
    // triangles outside and to each other.
    fresh.clear();
    for (int u : cavity) {
      for (int k = 0; k < 3; ++k) {
        const int o = tris[u].nb[k];
        if (o >= 0 && mark[o] == i) continue;
        const int a = tris[u].v[(k + 1) % 3], b = tris[u].v[(k + 2) % 3];
        const int nt = make(a, b, i);
        mark.push_back(-1);
        tris[nt].nb[2] = o;
        if (o >= 0)
          for (int m = 0; m < 3; ++m)
            if (tris[o].v[(m + 1) % 3] == b && tris[o].v[(m + 2) % 3] == a) tris[o].nb[m] = nt;
        first_of[a] = nt;
        last_of[b] = nt;
        fresh.push_back(nt);
      }
    }
    for (int u : cavity) tris[u].alive = false;
    for (int nt : fresh) {
      T& c = tris[nt];  // (a, b, i): across (b, i) starts at b, across (i, a) ends at a
      c.nb[0] = first_of[c.v[1]];
      c.nb[1] = last_of[c.v[0]];
    }
    for (int nt : fresh) first_of[tris[nt].v[0]] = last_of[tris[nt].v[1]] = -1;
    if (!fresh.empty()) last = fresh.back();
  }
  for (const T& t : tris) {
    if (!t.alive || t.v[0] >= n || t.v[1] >= n || t.v[2] >= n) continue;
    int v[3] = {t.v[0], t.v[1], t.v[2]};
    std::sort(v, v + 3);
    out.push_back(Tri{v[0], v[1], v[2]});
  }
  std::sort(out.begin(), out.end(), [](const Tri& p, const Tri& q) {
    return p.a != q.a ? p.a < q.a : (p.b != q.b ? p.b < q.b : p.c < q.c);
  });
  return out;
}

// ComputeSfMPlanarPrior (estimator.cc:664-940) at one level: the SfM points
// projected into the reference (K of this level), a Delaunay triangulation
// of their pixels, a plane per triangle through its three camera-frame
// points (the triangle skipped across a depth ratio above 1.5 or over 20000
// px^2), the triangles rasterised in order with the reference's parametric
// loop, and the pixels whose prior depth lies in the range.  The plane is
// the unit normal of the two edge vectors' cross product with d >= 0 (the
// reference takes the SVD null vector of the 3 x 4 system: the same plane).
// Returns false when fewer than 4 points project.
static bool sfm_prior(const ARef& ref, const double* K, int w, int h, std::vector<float4>& planes,
                      std::vector<unsigned>& mask) {
  const float fx = (float)K[0], fy = (float)K[4], cx = (float)K[2], cy = (float)K[5];
  const double* R = ref.views[0].R;
  const double* t = ref.views[0].t;
  struct Proj {
    float u, v, depth, cam[3];
  };
  std::vector<Proj> pr;
  const size_t n = ref.sfm.size() / 3;
  for (size_t i = 0; i < n; ++i) {
    const double* X = &ref.sfm[3 * i];
    double c[3];
    for (int r = 0; r < 3; ++r) c[r] = ((R[3 * r] * X[0] + R[3 * r + 1] * X[1]) + R[3 * r + 2] * X[2]) + t[r];
    if (c[2] <= 0.0) continue;
    const float depth = (float)c[2];
    if (depth < ref.depth_min || depth > ref.depth_max) continue;
    const float u = (float)((double)fx * (c[0] / c[2]) + (double)cx);
    const float v = (float)((double)fy * (c[1] / c[2]) + (double)cy);
    if (u < 0.0f || u >= (float)w || v < 0.0f || v >= (float)h) continue;
    pr.push_back(Proj{u, v, depth, {(float)c[0], (float)c[1], (float)c[2]}});
  }
  planes.assign((size_t)w * h, make_float4(0.0f, 0.0f, -1.0f, 0.0f));
  mask.assign((size_t)w * h, 0u);
  if (pr.size() < 4) return false;
  std::vector<double> px(pr.size()), py(pr.size());
  for (size_t i = 0; i < pr.size(); ++i) {
    px[i] = pr[i].u;
    py[i] = pr[i].v;
  }
  const std::vector<Tri> tris = delaunay(px, py, w, h);
  // The vertex lookup keys on the integer pixel; the last point wins.
  std::vector<int> key_to(pr.size());
  std::vector<std::pair<long long, int>> keys;
  for (size_t i = 0; i < pr.size(); ++i) keys.emplace_back((long long)(int)pr[i].v * w + (int)pr[i].u, (int)i);
  auto lookup = [&](long long k) {
    int best = -1;
    for (const auto& kv : keys)
      if (kv.first == k) best = kv.second;
    return best;
  };
  struct TriPlane {
    int x[3], y[3];
    float4 plane;
  };
  std::vector<TriPlane> kept;
  for (const Tri& tr : tris) {
    const int id[3] = {tr.a, tr.b, tr.c};
    TriPlane tp;
    int src[3];
    bool ok = true;
    for (int k = 0; k < 3; ++k) {
      tp.x[k] = (int)pr[id[k]].u;
      tp.y[k] = (int)pr[id[k]].v;
      if (tp.x[k] < 0 || tp.x[k] >= w || tp.y[k] < 0 || tp.y[k] >= h) ok = false;
      src[k] = ok ? lookup((long long)tp.y[k] * w + tp.x[k]) : -1;
      if (src[k] < 0) ok = false;
    }
    if (!ok) continue;
    const float d1 = pr[src[0]].depth, d2 = pr[src[1]].depth, d3 = pr[src[2]].depth;
    const float dmin = std::min(d1, std::min(d2, d3)), dmax = std::max(d1, std::max(d2, d3));
    if (dmin > 0.0f && dmax / dmin > 1.5f) continue;
    const float ax = (float)(tp.x[1] - tp.x[0]), ay = (float)(tp.y[1] - tp.y[0]);
    const float bx = (float)(tp.x[2] - tp.x[0]), by = (float)(tp.y[2] - tp.y[0]);
    if (0.5f * std::fabs(ax * by - ay * bx) > 20000.0f) continue;
    const float* P1 = pr[src[0]].cam;
    const float* P2 = pr[src[1]].cam;
    const float* P3 = pr[src[2]].cam;
    const float e1[3] = {P2[0] - P1[0], P2[1] - P1[1], P2[2] - P1[2]};
    const float e2[3] = {P3[0] - P1[0], P3[1] - P1[1], P3[2] - P1[2]};
    float nn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                   e1[0] * e2[1] - e1[1] * e2[0]};
    const float len = std::sqrt((nn[0] * nn[0] + nn[1] * nn[1]) + nn[2] * nn[2]);
    if (!(len > 0.0f)) continue;
    for (int k = 0; k < 3; ++k) nn[k] = nn[k] / len;
    float d = -((nn[0] * P1[0] + nn[1] * P1[1]) + nn[2] * P1[2]);
    if (1.0f / std::sqrt(1.0f + d * d) < 1e-8f) continue;
    if (d < 0.0f) {
      for (int k = 0; k < 3; ++k) nn[k] = -nn[k];
      d = -d;
    }
    tp.plane = make_float4(nn[0], nn[1], nn[2], d);
    kept.push_back(tp);
  }
  std::vector<int> tri_at((size_t)w * h, 0);
  for (size_t ti = 0; ti < kept.size(); ++ti) {
    const TriPlane& tp = kept[ti];
    const float l01 = std::hypot((float)(tp.x[0] - tp.x[1]), (float)(tp.y[0] - tp.y[1]));
    const float l02 = std::hypot((float)(tp.x[0] - tp.x[2]), (float)(tp.y[0] - tp.y[2]));
    const float l12 = std::hypot((float)(tp.x[1] - tp.x[2]), (float)(tp.y[1] - tp.y[2]));
    const float max_edge = std::max(l01, std::max(l02, l12));
    if (max_edge < 1.0f) continue;
    const float step = 1.0f / max_edge;
    for (float p = 0.0f; p < 1.0f; p += step)
      for (float q = 0.0f; q < 1.0f - p; q += step) {
        const int xx = (int)(p * (float)tp.x[0] + q * (float)tp.x[1] + (1.0f - p - q) * (float)tp.x[2]);
        const int yy = (int)(p * (float)tp.y[0] + q * (float)tp.y[1] + (1.0f - p - q) * (float)tp.y[2]);
        if (xx >= 0 && xx < w && yy >= 0 && yy < h) tri_at[(size_t)yy * w + xx] = (int)ti + 1;
      }
  }
  bool any = false;
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const size_t i = (size_t)y * w + x;
      if (!tri_at[i]) continue;
      const float4 pl = kept[tri_at[i] - 1].plane;
      const float r0 = ((float)x - cx) / fx, r1 = ((float)y - cy) / fy;
      const float den = (pl.x * r0 + pl.y * r1) + pl.z * 1.0f;
      const float d = std::fabs(den) > 1e-6f ? -pl.w / den : 0.0f;
      if (d >= ref.depth_min && d <= ref.depth_max) {
        planes[i] = pl;
        mask[i] = 1u;
        any = true;
      }
    }
  return any;
}

// A view at one pyramid level (BuildImagePyramid, estimator.cc:562-588).
struct LevelView {
  int W, H;
  const uint8_t* img;
  std::vector<uint8_t> scaled;
  double K[9];
};

static dn_status level_view(const AView& v, float scale, LevelView* out) {
  std::memcpy(out->K, v.K, sizeof(out->K));
  if (!(scale < 0.999f)) {
    out->W = v.W;
    out->H = v.H;
    out->img = v.img.data();
    return DN_OK;
  }
  const int nw = std::max((int)((float)v.W * scale), 1), nh = std::max((int)((float)v.H * scale), 1);
  const int k = v.W / nw;
  out->W = nw;
  out->H = nh;
  out->scaled.resize((size_t)nw * nh);
  if (nw * k == v.W && nh * k == v.H && v.H / nh == k)
    resize_area_u8(v.img.data(), v.W, v.H, k, out->scaled.data());  // integer ratio
  else
    resize_area_general_u8(v.img.data(), v.W, v.H, out->scaled.data(), nw, nh);
  out->img = out->scaled.data();
  const float sx = (float)nw / (float)v.W, sy = (float)nh / (float)v.H;
  out->K[0] *= (double)sx;
  out->K[2] *= (double)sx;
  out->K[4] *= (double)sy;
  out->K[5] *= (double)sy;
  return DN_OK;
}

// The coarser level's result of one reference: what UpsampleDepthNormal
// starts from.
struct Coarse {
  int W = 0, H = 0;
  std::vector<float> depth, normal, cost;
};

// RunLevel (estimator.cc:159-243) for one reference: pyramid images, random
// initialisation or upsampling from `coarse`, previous-level depths of the
// linked sources, the iterations and the readback (with the median only on
// the last level).  The result goes to ref.depth / normal / cost / conf.
// The device work runs on stream s between events ev0 and ev1.
static dn_status run_level(dn_acmmp* e, ARef& ref, int level, int n_levels, const Coarse* coarse,
                           const std::vector<std::pair<int, const Coarse*>>& prev, cudaStream_t s,
                           cudaEvent_t ev0, cudaEvent_t ev1) {
  const int nv = (int)ref.views.size();
  ACHECK(nv >= 2, "a reference view needs at least one source view");
  const int n_img = std::min(nv, 1 + kMaxSrc);
  struct StreamScope {
    cudaStream_t old;
    explicit StreamScope(cudaStream_t s) : old(tl_stream) { tl_stream = s; }
    ~StreamScope() { tl_stream = old; }
  } scope(s);
  const float scale = (float)(1.0 / std::pow(2.0, n_levels - 1 - level));
  std::vector<std::unique_ptr<DBuf<float>>> imgs;
  AScene S{};
  for (int i = 0; i < n_img; ++i) {
    LevelView lv;
    dn_status st = level_view(ref.views[i], scale, &lv);
    if (st != DN_OK) return st;
    // cv::Mat::convertTo(CV_32F, 1/255): float(v) * float(1/255).
    std::vector<float> f((size_t)lv.W * lv.H);
    const float sc = (float)(1.0 / 255.0);
    for (size_t k = 0; k < f.size(); ++k) f[k] = (float)lv.img[k] * sc;
    imgs.emplace_back(new DBuf<float>());
    ACUDA(imgs.back()->alloc(f.size()));
    ACUDA(cudaMemcpyAsync(imgs.back()->p, f.data(), f.size() * sizeof(float),
                          cudaMemcpyHostToDevice, s));
    ACUDA(cudaStreamSynchronize(s));  // f is released at the end of this iteration
    S.img[i] = AImg{imgs.back()->p, lv.W, lv.H};
    for (int k = 0; k < 9; ++k) {
      S.cam[i].K[k] = (float)lv.K[k];
      S.cam[i].R[k] = (float)ref.views[i].R[k];
    }
    for (int k = 0; k < 3; ++k) S.cam[i].t[k] = (float)ref.views[i].t[k];
  }
  const int W = S.img[0].W, H = S.img[0].H;
  S.W = W;
  S.H = H;
  S.n_src = n_img - 1;
  S.half_patch = e->patch_size / 2;
  S.top_k = e->top_k;
  S.sigma_spatial = e->sigma_spatial;
  S.sigma_color = e->sigma_color;
  S.census_weight = e->census_weight;
  S.smooth_weight = e->smooth_weight;
  S.geom_weight = e->geom_weight;
  S.depth_min = ref.depth_min;
  S.depth_max = ref.depth_max;
  const size_t npix = (size_t)W * H;
  // ComputeSfMPlanarPrior at this level's size and K.
  DBuf<float4> d_prior;
  DBuf<unsigned> d_pmask;
  S.prior_planes = nullptr;
  S.prior_mask = nullptr;
  if (!ref.sfm.empty()) {
    LevelView lv0;
    dn_status st0 = level_view(ref.views[0], scale, &lv0);
    if (st0 != DN_OK) return st0;
    std::vector<float4> hp;
    std::vector<unsigned> hm;
    if (sfm_prior(ref, lv0.K, W, H, hp, hm)) {
      ACUDA(d_prior.alloc(npix));
      ACUDA(d_pmask.alloc(npix));
      ACUDA(cudaMemcpyAsync(d_prior.p, hp.data(), npix * sizeof(float4), cudaMemcpyHostToDevice, s));
      ACUDA(cudaMemcpyAsync(d_pmask.p, hm.data(), npix * sizeof(unsigned), cudaMemcpyHostToDevice, s));
      ACUDA(cudaStreamSynchronize(s));
      S.prior_planes = d_prior.p;
      S.prior_mask = d_pmask.p;
    }
  }
  // UploadPreviousDepths (estimator.cc:56-106).
  DBuf<float> d_prev;
  S.prev = nullptr;
  S.prev_mask = 0u;
  if (!prev.empty() && e->geom_weight > 0.0f) {
    std::vector<float> flat((size_t)kMaxSrc * npix, 0.0f);
    for (const auto& pe : prev) {
      const int si = pe.first;
      if (si < 0 || si >= kMaxSrc) continue;
      const Coarse& c = *pe.second;
      float* dst = flat.data() + (size_t)si * npix;
      if (c.W != W || c.H != H)
        resize_linear_f32(c.depth.data(), c.W, c.H, dst, W, H);
      else
        std::memcpy(dst, c.depth.data(), npix * sizeof(float));
      S.prev_mask |= 1u << si;
    }
    ACUDA(d_prev.alloc(flat.size()));
    ACUDA(cudaMemcpyAsync(d_prev.p, flat.data(), flat.size() * sizeof(float),
                          cudaMemcpyHostToDevice, s));
    ACUDA(cudaStreamSynchronize(s));
    S.prev = d_prev.p;
  }
  DBuf<AScene> dS;
  DBuf<float4> planes, src_planes;
  DBuf<float> costs, depth, normal, cost, depth2;
  DBuf<uint2> rs;
  DBuf<unsigned> sel;
  ACUDA(dS.alloc(1));
  ACUDA(planes.alloc(npix));
  ACUDA(costs.alloc(npix));
  ACUDA(rs.alloc(npix));
  ACUDA(sel.alloc(npix));
  ACUDA(depth.alloc(npix));
  ACUDA(depth2.alloc(npix));
  ACUDA(normal.alloc(3 * npix));
  ACUDA(cost.alloc(npix));
  ACUDA(cudaMemcpyAsync(dS.p, &S, sizeof(S), cudaMemcpyHostToDevice, s));
  AState st{planes.p, costs.p, rs.p, sel.p};
  const dim3 blk(16, 8), grid((W + 15) / 16, (H + 7) / 8);
  const dim3 pblk(16, 4), pgrid(((W + 1) / 2 + 15) / 16, (H + 3) / 4);
  // Two warps per block, each with its NCC queue (at most 35.6 KB).
  const size_t pm_smem = 2 * sizeof(float) * (size_t)acm_queue_words(S.n_src);
  std::vector<float4> hsrc;
  if (coarse) {
    // UpsampleDepthNormal's host part (estimator.cc:600-640): coarse
    // (depth, normal) -> planes, with the fine K scaled to the coarse size.
    const ACam& c0 = S.cam[0];
    const int sw = coarse->W, sh = coarse->H;
    const float fx = c0.K[0] * (float)sw / (float)W, fy = c0.K[4] * (float)sh / (float)H;
    const float cxs = c0.K[2] * (float)sw / (float)W, cys = c0.K[5] * (float)sh / (float)H;
    hsrc.resize((size_t)sw * sh);
    for (int y = 0; y < sh; ++y)
      for (int x = 0; x < sw; ++x) {
        const size_t i = (size_t)y * sw + x;
        const float d = coarse->depth[i];
        const float* n = &coarse->normal[3 * i];
        const float p0 = d * ((float)x - cxs) / fx, p1 = d * ((float)y - cys) / fy, p2 = d;
        hsrc[i] = make_float4(n[0], n[1], n[2], -((n[0] * p0 + n[1] * p1) + n[2] * p2));
      }
    ACUDA(src_planes.alloc(hsrc.size()));
    ACUDA(cudaMemcpyAsync(src_planes.p, hsrc.data(), hsrc.size() * sizeof(float4),
                          cudaMemcpyHostToDevice, s));
  }
  ACUDA(cudaEventRecord(ev0, s));
  if (coarse)
    acm_upsample_kernel<<<grid, blk, 0, s>>>(dS.p, st, src_planes.p, coarse->W, coarse->H);
  else
    acm_init_kernel<<<grid, blk, 0, s>>>(dS.p, st);
  for (int it = 0; it < e->max_iterations; ++it) {
    acm_pm_kernel<<<pgrid, pblk, pm_smem, s>>>(dS.p, st, 0, it);
    acm_pm_kernel<<<pgrid, pblk, pm_smem, s>>>(dS.p, st, 1, it);
    acm_filter_kernel<<<pgrid, pblk, 0, s>>>(dS.p, st, 0);
    acm_filter_kernel<<<pgrid, pblk, 0, s>>>(dS.p, st, 1);
  }
  acm_readback_kernel<<<grid, blk, 0, s>>>(dS.p, st, depth.p, normal.p, cost.p);
  const bool last = level == n_levels - 1;
  if (last) acm_median_kernel<<<grid, blk, 0, s>>>(W, H, depth.p, depth2.p);
  ACUDA(cudaGetLastError());
  ACUDA(cudaEventRecord(ev1, s));
  ref.W = W;
  ref.H = H;
  ref.depth.resize(npix);
  ref.normal.resize(3 * npix);
  ref.cost.resize(npix);
  ref.conf.assign(npix, 0.0f);
  ACUDA(cudaMemcpyAsync(ref.depth.data(), last ? depth2.p : depth.p, npix * sizeof(float),
                        cudaMemcpyDeviceToHost, s));
  ACUDA(cudaMemcpyAsync(ref.normal.data(), normal.p, 3 * npix * sizeof(float),
                        cudaMemcpyDeviceToHost, s));
  ACUDA(cudaMemcpyAsync(ref.cost.data(), cost.p, npix * sizeof(float), cudaMemcpyDeviceToHost, s));
  ACUDA(cudaStreamSynchronize(s));
  return DN_OK;
}

// Run (cluster_estimator.cc:82-138): levels outermost, references in turn.
// A reference's previous-level depths for the geometric term come from the
// linked references' latest results: those of this level for references
// already done, of the last level for the rest, as in the reference.  That
// order matters only when a level uses previous depths; otherwise the
// references of a level are independent and run concurrently, each on its
// own stream (up to 8 at a time).  last_ms sums, over the levels, the device
// time: the span from the first reference's start to the last one's end
// where they run concurrently, the sum of their spans where they run in
// turn (the host work between them is not device time).
extern "C" dn_status dn_acmmp_run(dn_acmmp* e) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e, "NULL estimator");
  if (e->refs.empty()) return afail(DN_INVALID_ARG, "DepthmapClusterEstimator: no reference views");
  ACUDA(cudaSetDevice(e->device));
  e->last_ms = 0.0f;
  const int n_levels = std::max(1, e->hierarchy_levels);
  const int n_refs = (int)e->refs.size();
  std::vector<Coarse> latest(n_refs);  // each reference's latest intermediate result
  const int n_par = std::min(n_refs, 8);
  std::vector<cudaStream_t> streams(n_par, nullptr);
  std::vector<cudaEvent_t> ev0(n_refs, nullptr), ev1(n_refs, nullptr);
  cudaEvent_t eref = nullptr;
  struct Cleanup {
    std::vector<cudaStream_t>& s;
    std::vector<cudaEvent_t>& a;
    std::vector<cudaEvent_t>& b;
    cudaEvent_t& r;
    ~Cleanup() {
      for (auto x : s)
        if (x) cudaStreamDestroy(x);
      for (auto x : a)
        if (x) cudaEventDestroy(x);
      for (auto x : b)
        if (x) cudaEventDestroy(x);
      if (r) cudaEventDestroy(r);
    }
  } cleanup{streams, ev0, ev1, eref};
  for (auto& x : streams) ACUDA(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
  for (int i = 0; i < n_refs; ++i) {
    ACUDA(cudaEventCreate(&ev0[i]));
    ACUDA(cudaEventCreate(&ev1[i]));
  }
  ACUDA(cudaEventCreate(&eref));

  auto links_of = [&](int i) {
    std::vector<std::pair<int, const Coarse*>> prev;
    for (size_t l = 0; l + 2 < e->geom_links.size(); l += 3)
      if (e->geom_links[l] == i) {
        const int fr = e->geom_links[l + 2];
        if (fr >= 0 && fr < n_refs && !latest[fr].depth.empty())
          prev.emplace_back(e->geom_links[l + 1], &latest[fr]);
      }
    return prev;
  };
  auto keep = [&](int i, int level) {
    if (level < n_levels - 1) {
      const ARef& ref = e->refs[i];
      latest[i].W = ref.W;
      latest[i].H = ref.H;
      latest[i].depth = ref.depth;
      latest[i].normal = ref.normal;
      latest[i].cost = ref.cost;
    }
  };

  for (int level = 0; level < n_levels; ++level) {
    const bool uses_prev = level > 0 && e->geom_weight > 0.0f && !e->geom_links.empty();
    ACUDA(cudaEventRecord(eref, e->stream));
    ACUDA(cudaStreamSynchronize(e->stream));
    if (uses_prev) {
      for (int i = 0; i < n_refs; ++i) {
        Coarse own = latest[i];  // a copy: latest[i] is replaced below
        const dn_status st = run_level(e, e->refs[i], level, n_levels, level > 0 ? &own : nullptr,
                                       links_of(i), streams[0], ev0[i], ev1[i]);
        if (st != DN_OK) return st;
        keep(i, level);
      }
    } else {
      const std::vector<Coarse> own = latest;  // the upsampling inputs of this level
      std::vector<dn_status> sts(n_refs, DN_OK);
      std::vector<std::string> msgs(n_refs);
      for (int i0 = 0; i0 < n_refs; i0 += n_par) {
        std::vector<std::thread> pool;
        for (int i = i0; i < std::min(n_refs, i0 + n_par); ++i)
          pool.emplace_back([&, i]() {
            cudaSetDevice(e->device);
            const std::vector<std::pair<int, const Coarse*>> none;
            sts[i] = run_level(e, e->refs[i], level, n_levels, level > 0 ? &own[i] : nullptr,
                               none, streams[i - i0], ev0[i], ev1[i]);
            if (sts[i] != DN_OK) msgs[i] = g_acm_error;
          });
        for (auto& t : pool) t.join();
      }
      for (int i = 0; i < n_refs; ++i)
        if (sts[i] != DN_OK) return afail(sts[i], msgs[i]);
      for (int i = 0; i < n_refs; ++i) keep(i, level);
    }
    float t_first = 0.0f, t_last = 0.0f, t_sum = 0.0f;
    for (int i = 0; i < n_refs; ++i) {
      float a = 0.0f, b = 0.0f;
      ACUDA(cudaEventElapsedTime(&a, eref, ev0[i]));
      ACUDA(cudaEventElapsedTime(&b, eref, ev1[i]));
      t_first = i == 0 ? a : std::min(t_first, a);
      t_last = i == 0 ? b : std::max(t_last, b);
      t_sum += b - a;
    }
    e->last_ms += uses_prev ? t_sum : t_last - t_first;
  }
  // Logistic confidence on the host, as the reference computes it
  // (estimator.cc:1023-1037).
  for (auto& ref : e->refs)
    for (size_t i = 0; i < ref.depth.size(); ++i)
      if (ref.depth[i] > 0.0f) ref.conf[i] = 1.0f / (1.0f + std::exp((ref.cost[i] - 0.5f) * 5.0f));
  return DN_OK;
}

extern "C" dn_status dn_acmmp_result_size(dn_acmmp* e, int ref_idx, int* w, int* h) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e && w && h, "NULL argument");
  if (ref_idx < 0 || ref_idx >= (int)e->refs.size()) return afail(DN_OUT_OF_RANGE, "ref index out of range");
  *w = e->refs[ref_idx].W ? e->refs[ref_idx].W : e->refs[ref_idx].views[0].W;
  *h = e->refs[ref_idx].H ? e->refs[ref_idx].H : e->refs[ref_idx].views[0].H;
  return DN_OK;
}

extern "C" dn_status dn_acmmp_get_result(dn_acmmp* e, int ref_idx, float* depth, float* normal,
                                         float* cost, float* confidence) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e, "NULL estimator");
  if (ref_idx < 0 || ref_idx >= (int)e->refs.size()) return afail(DN_OUT_OF_RANGE, "ref index out of range");
  const ARef& r = e->refs[ref_idx];
  ACHECK(!r.depth.empty(), "run() has not produced this result");
  if (depth) std::memcpy(depth, r.depth.data(), r.depth.size() * sizeof(float));
  if (normal) std::memcpy(normal, r.normal.data(), r.normal.size() * sizeof(float));
  if (cost) std::memcpy(cost, r.cost.data(), r.cost.size() * sizeof(float));
  if (confidence) std::memcpy(confidence, r.conf.data(), r.conf.size() * sizeof(float));
  return DN_OK;
}

extern "C" dn_status dn_acmmp_last_run_ms(dn_acmmp* e, float* ms) {
  const dn::DeviceRestore device_restore_;
  ACHECK(e && ms, "NULL argument");
  *ms = e->last_ms;
  return DN_OK;
}

extern "C" dn_status dn_delaunay_2d(const double* xy, int n, int w, int h, int* tris, int capacity,
                                     int* count) {
  const dn::DeviceRestore device_restore_;
  ACHECK(count && (n == 0 || xy) && n >= 0 && w > 0 && h > 0, "bad argument");
  for (int i = 0; i < 2 * n; ++i) ACHECK(std::isfinite(xy[i]), "non-finite coordinate");
  std::vector<double> px(n), py(n);
  for (int i = 0; i < n; ++i) {
    px[i] = xy[2 * i];
    py[i] = xy[2 * i + 1];
  }
  const std::vector<Tri> t = delaunay(px, py, w, h);
  *count = (int)t.size();
  ACHECK(!tris || capacity >= (int)t.size(), "capacity below the triangle count");
  if (tris)
    for (size_t i = 0; i < t.size(); ++i) {
      tris[3 * i] = t[i].a;
      tris[3 * i + 1] = t[i].b;
      tris[3 * i + 2] = t[i].c;
    }
  return DN_OK;
}
