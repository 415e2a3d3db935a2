// Device-side data layout and helpers shared by the dense kernels.
//
// HBM layout (one reconstruction = a set of views + a set of depthmaps):
//   ViewDev  per view:  FP16 image [H][W] (uint8 intensities are exact in
//            FP16), optional uint8 mask, and a bilinear coefficient table
//            `quad` [(H-1+2P)][(W-1+2P)] of float4 (see build_quad_kernel).
//   PairDev  per (depthmap, matching view): the plane-induced homography
//            split as H(v) = G + e f^T with G = K_o Q_o K_0^-1, e = K_o a_o,
//            f = K_0^-T v (reference depthmap.cc:88-102 composes the same
//            matrix as K_o (Q_o + a_o v^T) K_0^-1), built in FP64 on the host.
//   MapDev   per depthmap: state float4 [H][W] = (plane v, depth), score f32,
//            nghbr i32, plus the outputs.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace dn {

constexpr int kPad = 8;        // zero border of the coefficient tables (pixels)
constexpr int kMaxNbr = 16;    // matching views per depthmap
constexpr int kMaxHpz = 5;     // patch half-size supported (patch 3..11)
constexpr int kFarSamples = 11;  // far propagation samples per direction
constexpr int kFarStart = 3;     // first far sample distance (then +2)

struct ViewDev {
  const __half* img;     // [H][W]
  const uint8_t* mask;   // [H][W] or null (all valid)
  const float4* quad;    // [TH][TW]
  int W, H, TW, TH;
  float cbias;           // intensity centring constant folded into quad.x
  int pad_[3];
};

struct PairDev {
  float G[9];
  float e[3];
  int view;
  int pad_[3];
};

struct MapDev {
  int ref_view, W, H, n_pairs;
  int pair0, clean0, n_clean, prune_off;  // clean0: offset in clean list
  float Kinv[9];                           // FP32 copy of K_0^-1
  float log_min, log_max;                  // log depth range (init)
  double Kinv_d[9];                        // FP64 K_0^-1 (plane/depth conversions)
  double min_depth, max_depth;             // brute-force sweep range
  double K[9], R[9], t[3];                 // FP64 camera (cleaner / pruner)
  float4* state;                           // [H][W] (v.x, v.y, v.z, depth)
  float* score;                            // [H][W]
  int* nghbr;                              // [H][W]
  float* depth;                            // [H][W] final (post-processed) depth
  float* clean;                            // [H][W] cleaned depth
  const float* init;                       // [H][W][3] optional initial planes
  uint8_t* keep;                           // [H][W] pruner flags (scratch)
};

struct RunParams {
  int hpz;
  float min_var;       // min patch variance (sd^2)
  uint32_t seed_lo, seed_hi;
  int num_planes;
  int colour;          // red-black colour of this half-pass
  int pass;            // half-pass counter (RNG stream)
  float same_depth_thr;
  int min_consistent;
  unsigned long long* taps;  // NCC tap counter
  int* error;                // device error word
  int variant;               // NCC walk: 0/1 one view at a time, 2/3 views in lock step
};

// ------------------------------------------------------------------ RNG
// Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with the
// published multipliers and Weyl key increments.
__host__ __device__ inline uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}
__host__ __device__ inline uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = mulhi32(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = mulhi32(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
  }
  return c;
}
// Uniform in [0, 1) with 24 random bits.
__device__ inline float u01(uint32_t x) { return (x >> 8) * (1.0f / 16777216.0f); }
// Box-Muller pair of standard normals from two 32-bit draws.
__device__ inline float2 normal2(uint32_t a, uint32_t b) {
  const float u1 = ((a >> 8) + 1) * (1.0f / 16777216.0f);  // (0, 1]
  const float r = sqrtf(-2.0f * logf(u1));
  float s, c;
  sincospif(2.0f * u01(b), &s, &c);
  return make_float2(r * c, r * s);
}

// ------------------------------------------------------- exact helpers
// Round-to-nearest products and sums that the compiler may not contract,
// so these follow the reference's double/float evaluation order exactly.
__device__ inline double dot3_rn(const double* a, double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(a[0], x), __dmul_rn(a[1], y)), __dmul_rn(a[2], z));
}

// PlaneFromDepthAndNormal (depthmap.cc:120-125): X = (float)((depth K^-1) q),
// v = n * (1 / max(1e-6, -n.X)) in float.
__device__ inline float3 plane_from_depth_normal(float x, float y, const double* Kinv,
                                                 float depth, float3 n) {
  const double d = (double)depth;
  double M[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) M[k] = __dmul_rn(Kinv[k], d);
  const float px = (float)dot3_rn(M + 0, x, y, 1.0);
  const float py = (float)dot3_rn(M + 3, x, y, 1.0);
  const float pz = (float)dot3_rn(M + 6, x, y, 1.0);
  const float s = __fadd_rn(__fadd_rn(__fmul_rn(n.x, px), __fmul_rn(n.y, py)), __fmul_rn(n.z, pz));
  const float denom = -s;
  const float m = (1e-6f < denom) ? denom : 1e-6f;
  const float inv = __frcp_rn(m);
  return make_float3(__fmul_rn(n.x, inv), __fmul_rn(n.y, inv), __fmul_rn(n.z, inv));
}

// DepthOfPlaneBackprojection (depthmap.cc:114-118): 1 / max(1e-6,
// -(v^T K^-1 q)) with the row vector v^T K^-1 formed first, in double.
__device__ inline float depth_of_plane(double x, double y, const double* Kinv, float3 v) {
  double r[3];
#pragma unroll
  for (int j = 0; j < 3; ++j)
    r[j] = __dadd_rn(__dadd_rn(__dmul_rn((double)v.x, Kinv[j]), __dmul_rn((double)v.y, Kinv[3 + j])),
                     __dmul_rn((double)v.z, Kinv[6 + j]));
  const double s = __dadd_rn(__dadd_rn(__dmul_rn(r[0], x), __dmul_rn(r[1], y)), r[2]);
  const float denom = (float)(-s);
  const float m = (1e-6f < denom) ? denom : 1e-6f;
  return __fdiv_rn(1.0f, m);
}

__device__ inline bool same_plane(float3 a, float3 b) {
  return __float_as_uint(a.x) == __float_as_uint(b.x) &&
         __float_as_uint(a.y) == __float_as_uint(b.y) &&
         __float_as_uint(a.z) == __float_as_uint(b.z);
}

// ------------------------------------------------------------ NCC core
// Reference-side patch terms, hoisted per pixel (depthmap.cc:467-476 and
// 480-487 recompute them for every hypothesis): bilateral weights w_t, the
// weighted mean-centred reference intensities w_t * (x_t - mean_x), and
// var_x.  NT = (2 HPZ + 1)^2 taps, kept in registers.
template <int HPZ>
struct RefPatch {
  static constexpr int N = (2 * HPZ + 1) * (2 * HPZ + 1);
  float w[N];
  float wx[N];
  float inv_sw;
  float varx;
};

// Builds the reference patch terms for pixel (i, j) from a float tile in
// shared memory (tile origin (ty0, tx0), row pitch `pitch`).
template <int HPZ>
__device__ inline void ref_patch_from_tile(RefPatch<HPZ>& rp, const float* tile, int pitch,
                                           int ly, int lx) {
  // ly, lx: tile coordinates of the centre pixel.
  const float c = tile[ly * pitch + lx];
  const float dcf = 1.0f / 5000.0f;  // 1 / (2 * 50^2)
  const float dxf = 1.0f / 50.0f;    // 1 / (2 * 5^2)
  float sw = 0.f, swx = 0.f;
  float xs[RefPatch<HPZ>::N];
#pragma unroll
  for (int dy = -HPZ; dy <= HPZ; ++dy)
#pragma unroll
    for (int dx = -HPZ; dx <= HPZ; ++dx) {
      const int t = (dy + HPZ) * (2 * HPZ + 1) + (dx + HPZ);
      const float x = tile[(ly + dy) * pitch + lx + dx];
      const float d = __fsub_rn(x, c);
      const float arg = __fsub_rn(__fmul_rn(__fmul_rn(-d, d), dcf),
                                  __fmul_rn((float)(dx * dx + dy * dy), dxf));
      const float w = expf(arg);
      rp.w[t] = w;
      xs[t] = x;
      sw += w;
      swx = fmaf(w, x, swx);
    }
  const float inv_sw = 1.0f / sw;
  const float mx = swx * inv_sw;
  float sxx = 0.f;
#pragma unroll
  for (int t = 0; t < RefPatch<HPZ>::N; ++t) {
    const float xc = xs[t] - mx;
    rp.wx[t] = rp.w[t] * xc;
    sxx = fmaf(rp.wx[t], xc, sxx);
  }
  rp.inv_sw = inv_sw;
  rp.varx = sxx * inv_sw;
}

// Per-hypothesis terms shared by every matching view: f = K_0^-T v and
// f.q for the pixel q = (j, i, 1).
struct Hyp {
  float f0, f1, fq;
};
__device__ inline Hyp make_hyp(const float* Kinv, float3 v, float j, float i) {
  Hyp h;
  h.f0 = fmaf(Kinv[0], v.x, fmaf(Kinv[3], v.y, Kinv[6] * v.z));
  h.f1 = fmaf(Kinv[1], v.x, fmaf(Kinv[4], v.y, Kinv[7] * v.z));
  const float f2 = fmaf(Kinv[2], v.x, fmaf(Kinv[5], v.y, Kinv[8] * v.z));
  h.fq = fmaf(h.f0, j, fmaf(h.f1, i, f2));
  return h;
}

// Local affine warp of the plane-induced homography at the patch centre
// (ComputePlaneImageScore, depthmap.cc:449-465): centre (X0, Y0) and the
// Jacobian columns (ax, ay) per dx and (bx, by) per dy, plus how the patch
// can be sampled: kOutside (every tap outside the image: all samples 0,
// var_y = 0, NCC = -1), kFast (inside the padded table, fixed-point path),
// kSlow (float coordinates, clamped), kDegenerate (w == 0: NCC = -1).
enum WarpMode { kOutside = 0, kFast = 1, kSlow = 2, kDegenerate = 3 };
struct Warp {
  float X0, Y0, ax, bx, ay, by;
  int mode;
};

template <int HPZ>
__device__ inline Warp warp_setup(const ViewDev& vw, const PairDev& pr, const Hyp& h, float j,
                                  float i) {
  Warp wp;
  const float gq0 = fmaf(pr.G[0], j, fmaf(pr.G[1], i, pr.G[2]));
  const float gq1 = fmaf(pr.G[3], j, fmaf(pr.G[4], i, pr.G[5]));
  const float gq2 = fmaf(pr.G[6], j, fmaf(pr.G[7], i, pr.G[8]));
  const float u = fmaf(pr.e[0], h.fq, gq0);
  const float v = fmaf(pr.e[1], h.fq, gq1);
  const float w = fmaf(pr.e[2], h.fq, gq2);
  if (w == 0.0f) {
    wp.mode = kDegenerate;
    wp.X0 = wp.Y0 = wp.ax = wp.bx = wp.ay = wp.by = 0.f;
    return wp;
  }
  const float H00 = fmaf(pr.e[0], h.f0, pr.G[0]), H01 = fmaf(pr.e[0], h.f1, pr.G[1]);
  const float H10 = fmaf(pr.e[1], h.f0, pr.G[3]), H11 = fmaf(pr.e[1], h.f1, pr.G[4]);
  const float H20 = fmaf(pr.e[2], h.f0, pr.G[6]), H21 = fmaf(pr.e[2], h.f1, pr.G[7]);
  const float rw = 1.0f / w;
  wp.X0 = u * rw;
  wp.Y0 = v * rw;
  wp.ax = (H00 - H20 * wp.X0) * rw;  // d x2 / d dx
  wp.bx = (H01 - H21 * wp.X0) * rw;  // d x2 / d dy
  wp.ay = (H10 - H20 * wp.Y0) * rw;  // d y2 / d dx
  wp.by = (H11 - H21 * wp.Y0) * rw;  // d y2 / d dy
  const float ex = HPZ * (fabsf(wp.ax) + fabsf(wp.bx));
  const float ey = HPZ * (fabsf(wp.ay) + fabsf(wp.by));
  const float Wm1 = (float)(vw.W - 1), Hm1 = (float)(vw.H - 1);
  if (wp.X0 + ex < -0.01f || wp.X0 - ex >= Wm1 + 0.01f || wp.Y0 + ey < -0.01f ||
      wp.Y0 - ey >= Hm1 + 0.01f) {
    wp.mode = kOutside;
    return wp;
  }
  const float lo = -(float)kPad + 0.01f;
  const bool fast = (wp.X0 - ex >= lo) && (wp.X0 + ex < Wm1 + (float)kPad - 0.01f) &&
                    (wp.Y0 - ey >= lo) && (wp.Y0 + ey < Hm1 + (float)kPad - 0.01f) &&
                    ex < 200.f && ey < 200.f;
  wp.mode = fast ? kFast : kSlow;
  return wp;
}

// Fixed-point walk of one view's patch: tap (dx, dy) sits at
// XS + dx AX + dy BX (9.23 fixed point, relative to floor(X0)), likewise y.
struct Walk {
  const float4* base;  // table entry of (floor(X0), floor(Y0))
  int XS, YS, AX, AY, BX, BY;
  int TW;
};

template <int HPZ>
__device__ inline Walk make_walk(const ViewDev& vw, const Warp& wp) {
  Walk k;
  const float fbx = floorf(wp.X0), fby = floorf(wp.Y0);
  const float sc = 8388608.0f;  // 2^23
  k.XS = __float2int_rn((wp.X0 - fbx - HPZ * wp.ax - HPZ * wp.bx) * sc);
  k.YS = __float2int_rn((wp.Y0 - fby - HPZ * wp.ay - HPZ * wp.by) * sc);
  k.AX = __float2int_rn(wp.ax * sc);
  k.BX = __float2int_rn(wp.bx * sc);
  k.AY = __float2int_rn(wp.ay * sc);
  k.BY = __float2int_rn(wp.by * sc);
  k.TW = vw.TW;
  k.base = vw.quad + (size_t)((int)fby + kPad) * vw.TW + ((int)fbx + kPad);
  return k;
}

// Sample of the coefficient table at fixed-point (XF, YF): the fraction
// bits become the float 1 + f directly; one 16-byte load and three FMAs.
__device__ inline float walk_sample(const Walk& k, int XF, int YF) {
  const int ix = XF >> 23, iy = YF >> 23;
  const float f1 = __int_as_float((XF & 0x7FFFFF) | 0x3F800000);
  const float g1 = __int_as_float((YF & 0x7FFFFF) | 0x3F800000);
  const float4 q = __ldg(k.base + iy * k.TW + ix);
  return fmaf(g1, fmaf(f1, q.w, q.z), fmaf(f1, q.y, q.x));
}

template <int HPZ>
__device__ inline float ncc_finish(const RefPatch<HPZ>& rp, float s1, float s2, float s3) {
  const float my = s1 * rp.inv_sw;
  const float vary = fmaf(s2, rp.inv_sw, -my * my);
  if (rp.varx < 0.1f || vary < 0.1f) return -1.0f;
  return (s3 * rp.inv_sw) * rsqrtf(rp.varx * vary);
}

// Slow path: float tap coordinates; out-of-table taps read the table's
// corner entry, whose sample is the reference's zero.
template <int HPZ>
__device__ inline float ncc_slow(const RefPatch<HPZ>& rp, const ViewDev& vw, const Warp& wp) {
  const float Wm1 = (float)(vw.W - 1), Hm1 = (float)(vw.H - 1);
  const float xlo = -(float)kPad, xhi = Wm1 + (float)kPad;
  const float ylo = -(float)kPad, yhi = Hm1 + (float)kPad;
  float s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
  for (int dy = -HPZ; dy <= HPZ; ++dy)
#pragma unroll
    for (int dx = -HPZ; dx <= HPZ; ++dx) {
      const float x = fmaf(wp.bx, (float)dy, fmaf(wp.ax, (float)dx, wp.X0));
      const float yv = fmaf(wp.by, (float)dy, fmaf(wp.ay, (float)dx, wp.Y0));
      int ix = -kPad, iy = -kPad;
      float f1 = 1.f, g1 = 1.f;
      if (x >= xlo && x < xhi && yv >= ylo && yv < yhi) {
        const float fx = floorf(x), fy = floorf(yv);
        ix = (int)fx;
        iy = (int)fy;
        f1 = 1.0f + (x - fx);
        g1 = 1.0f + (yv - fy);
      }
      const float4 q = __ldg(vw.quad + (size_t)(iy + kPad) * vw.TW + (ix + kPad));
      const float y = fmaf(g1, fmaf(f1, q.w, q.z), fmaf(f1, q.y, q.x));
      const int t = (dy + HPZ) * (2 * HPZ + 1) + (dx + HPZ);
      const float wy = rp.w[t] * y;
      s1 += wy;
      s2 = fmaf(wy, y, s2);
      s3 = fmaf(rp.wx[t], y, s3);
    }
  return ncc_finish<HPZ>(rp, s1, s2, s3);
}

// Bilateral NCC of the reference patch against one matching view under
// hypothesis h (ComputePlaneImageScore, depthmap.cc:441-478; NCCEstimator,
// depthmap.cc:46-74).  Same local affine warp of the plane-induced
// homography, same bilinear sample with zeros outside [0,W-1) x [0,H-1),
// same weights.  Sums are mean-centred: x by the patch's weighted mean
// (hoisted), y by the view's constant cbias (folded into the table).
template <int HPZ>
__device__ inline float ncc_view(const RefPatch<HPZ>& rp, const ViewDev& vw, const PairDev& pr,
                                 const Hyp& h, float j, float i, unsigned& taps) {
  const Warp wp = warp_setup<HPZ>(vw, pr, h, j, i);
  if (wp.mode == kOutside || wp.mode == kDegenerate) return -1.0f;
  taps += RefPatch<HPZ>::N;
  if (wp.mode == kSlow) return ncc_slow<HPZ>(rp, vw, wp);
  const Walk k = make_walk<HPZ>(vw, wp);
  float s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
  for (int dy = 0; dy <= 2 * HPZ; ++dy) {
    const int xr = k.XS + dy * k.BX, yr = k.YS + dy * k.BY;
#pragma unroll
    for (int dx = 0; dx <= 2 * HPZ; ++dx) {
      const float y = walk_sample(k, xr + dx * k.AX, yr + dx * k.AY);
      const int t = dy * (2 * HPZ + 1) + dx;
      const float wy = rp.w[t] * y;
      s1 += wy;
      s2 = fmaf(wy, y, s2);
      s3 = fmaf(rp.wx[t], y, s3);
    }
  }
  return ncc_finish<HPZ>(rp, s1, s2, s3);
}

// ComputePlaneScore (depthmap.cc:408-419): max over matching views, the
// first maximum wins, -1 / view 0 when every view fails.
template <int HPZ>
__device__ inline float ncc_max(const RefPatch<HPZ>& rp, const ViewDev* views,
                                const PairDev* pairs, int n_pairs, const Hyp& h, float j,
                                float i, int& best_view, unsigned& taps) {
  float best = -1.0f;
  best_view = 0;
  for (int k = 0; k < n_pairs; ++k) {
    const PairDev& pr = pairs[k];
    const float s = ncc_view<HPZ>(rp, views[pr.view], pr, h, j, i, taps);
    if (s > best) {
      best = s;
      best_view = k + 1;
    }
  }
  return best;
}

// ------------------------------------------------------------------------
// Cooperative 7 x 7 patch: L lanes (2 or 4, adjacent in the warp) share one
// pixel.  The patch is padded to 8 columns; lane l owns columns l, l + L,
// ... (8 / L columns x 7 rows), the padding column carries weight 0 and
// samples column 6's position.  Each lane keeps 2 x 56 / L weights instead of
// 98, so more warps fit on an SM, and lanes l and l + 1 read neighbouring
// table entries.  The three sums are combined with XOR shuffles inside the
// lane group; every lane of a group ends with the same score.
template <int L>
struct CoopPatch {
  static constexpr int C = 8 / L;  // columns per lane
  static constexpr int S = 7 * C;  // slots per lane
  float w[S];
  float wx[S];
  float inv_sw;
  float varx;
  int lane;
  unsigned mask;  // the lane group's bits in the warp
};

template <int L>
__device__ inline float group_sum(float v, unsigned mask) {
#pragma unroll
  for (int o = 1; o < L; o <<= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}

template <int L>
__device__ inline void coop_patch_from_tile(CoopPatch<L>& cp, const float* tile, int pitch, int ly,
                                            int lx, int lane, unsigned mask) {
  cp.lane = lane;
  cp.mask = mask;
  const float c = tile[ly * pitch + lx];
  const float dcf = 1.0f / 5000.0f;
  const float dxf = 1.0f / 50.0f;
  float sw = 0.f, swx = 0.f;
  float xs[CoopPatch<L>::S];
#pragma unroll
  for (int r = 0; r < 7; ++r)
#pragma unroll
    for (int q = 0; q < CoopPatch<L>::C; ++q) {
      const int t = r * CoopPatch<L>::C + q;
      const int dx = lane + L * q;
      const bool real = dx < 7;
      const int dxx = real ? dx : 6;
      const float x = tile[(ly + r - 3) * pitch + lx + dxx - 3];
      const float d = __fsub_rn(x, c);
      const int ddx = dxx - 3, ddy = r - 3;
      const float arg = __fsub_rn(__fmul_rn(__fmul_rn(-d, d), dcf),
                                  __fmul_rn((float)(ddx * ddx + ddy * ddy), dxf));
      const float w = real ? expf(arg) : 0.0f;
      cp.w[t] = w;
      xs[t] = x;
      sw += w;
      swx = fmaf(w, x, swx);
    }
  sw = group_sum<L>(sw, mask);
  swx = group_sum<L>(swx, mask);
  const float inv_sw = 1.0f / sw;
  const float mx = swx * inv_sw;
  float sxx = 0.f;
#pragma unroll
  for (int t = 0; t < CoopPatch<L>::S; ++t) {
    const float xc = xs[t] - mx;
    cp.wx[t] = cp.w[t] * xc;
    sxx = fmaf(cp.wx[t], xc, sxx);
  }
  sxx = group_sum<L>(sxx, mask);
  cp.inv_sw = inv_sw;
  cp.varx = sxx * inv_sw;
}

template <int L>
__device__ inline float coop_finish(const CoopPatch<L>& cp, float s1, float s2, float s3) {
  s1 = group_sum<L>(s1, cp.mask);
  s2 = group_sum<L>(s2, cp.mask);
  s3 = group_sum<L>(s3, cp.mask);
  const float my = s1 * cp.inv_sw;
  const float vary = fmaf(s2, cp.inv_sw, -my * my);
  if (cp.varx < 0.1f || vary < 0.1f) return -1.0f;
  return (s3 * cp.inv_sw) * rsqrtf(cp.varx * vary);
}

template <int L>
__device__ inline float coop_ncc_view(const CoopPatch<L>& cp, const ViewDev& vw,
                                      const PairDev& pr, const Hyp& h, float j, float i,
                                      unsigned& taps) {
  constexpr int C = CoopPatch<L>::C;
  const Warp wp = warp_setup<3>(vw, pr, h, j, i);
  if (wp.mode == kOutside || wp.mode == kDegenerate) return -1.0f;
  if (cp.lane == 0) taps += 49;
  // The padding column (dx = 7, on lane L - 1) samples dx = 6.
  const int pad_col = (cp.lane == L - 1) ? 1 : 0;
  float s1 = 0.f, s2 = 0.f, s3 = 0.f;
  if (wp.mode == kSlow) {
    const float Wm1 = (float)(vw.W - 1), Hm1 = (float)(vw.H - 1);
    const float xlo = -(float)kPad, xhi = Wm1 + (float)kPad;
    const float ylo = -(float)kPad, yhi = Hm1 + (float)kPad;
#pragma unroll
    for (int r = 0; r < 7; ++r)
#pragma unroll
      for (int q = 0; q < C; ++q) {
        const int dx = cp.lane + L * q - ((q == C - 1) ? pad_col : 0) - 3;
        const int dy = r - 3;
        const float x = fmaf(wp.bx, (float)dy, fmaf(wp.ax, (float)dx, wp.X0));
        const float yv = fmaf(wp.by, (float)dy, fmaf(wp.ay, (float)dx, wp.Y0));
        int ix = -kPad, iy = -kPad;
        float f1 = 1.f, g1 = 1.f;
        if (x >= xlo && x < xhi && yv >= ylo && yv < yhi) {
          const float fx = floorf(x), fy = floorf(yv);
          ix = (int)fx;
          iy = (int)fy;
          f1 = 1.0f + (x - fx);
          g1 = 1.0f + (yv - fy);
        }
        const float4 qd = __ldg(vw.quad + (size_t)(iy + kPad) * vw.TW + (ix + kPad));
        const float y = fmaf(g1, fmaf(f1, qd.w, qd.z), fmaf(f1, qd.y, qd.x));
        const int t = r * C + q;
        const float wy = cp.w[t] * y;
        s1 += wy;
        s2 = fmaf(wy, y, s2);
        s3 = fmaf(cp.wx[t], y, s3);
      }
  } else {
    const Walk k = make_walk<3>(vw, wp);
    const int xs = k.XS + cp.lane * k.AX, ys = k.YS + cp.lane * k.AY;
    const int xpad = pad_col * k.AX, ypad = pad_col * k.AY;
#pragma unroll
    for (int r = 0; r < 7; ++r) {
      const int xr = xs + r * k.BX, yr = ys + r * k.BY;
#pragma unroll
      for (int q = 0; q < C; ++q) {
        int XF = xr + (L * q) * k.AX, YF = yr + (L * q) * k.AY;
        if (q == C - 1) {
          XF -= xpad;
          YF -= ypad;
        }
        const float y = walk_sample(k, XF, YF);
        const int t = r * C + q;
        const float wy = cp.w[t] * y;
        s1 += wy;
        s2 = fmaf(wy, y, s2);
        s3 = fmaf(cp.wx[t], y, s3);
      }
    }
  }
  return coop_finish<L>(cp, s1, s2, s3);
}

// ------------------------------------------------------------------------
// One interface for both layouts: Patch<HPZ, L>.
template <int HPZ, int L>
struct Patch;

template <int HPZ>
struct Patch<HPZ, 1> {
  RefPatch<HPZ> rp;
  __device__ void build(const float* tile, int pitch, int ly, int lx, int, unsigned) {
    ref_patch_from_tile<HPZ>(rp, tile, pitch, ly, lx);
  }
  __device__ float view(const ViewDev& vw, const PairDev& pr, const Hyp& h, float j, float i,
                        unsigned& taps) const {
    return ncc_view<HPZ>(rp, vw, pr, h, j, i, taps);
  }
};

template <int L>
struct CoopIface {
  CoopPatch<L> cp;
  __device__ void build(const float* tile, int pitch, int ly, int lx, int lane, unsigned mask) {
    coop_patch_from_tile<L>(cp, tile, pitch, ly, lx, lane, mask);
  }
  __device__ float view(const ViewDev& vw, const PairDev& pr, const Hyp& h, float j, float i,
                        unsigned& taps) const {
    return coop_ncc_view<L>(cp, vw, pr, h, j, i, taps);
  }
};
template <>
struct Patch<3, 2> : CoopIface<2> {};
template <>
struct Patch<3, 4> : CoopIface<4> {};

template <int HPZ, int L>
__device__ inline float patch_max(const Patch<HPZ, L>& pt, const ViewDev* views,
                                  const PairDev* pairs, int n_pairs, const Hyp& h, float j,
                                  float i, int& best_view, unsigned& taps) {
  float best = -1.0f;
  best_view = 0;
  for (int k = 0; k < n_pairs; ++k) {
    const PairDev& pr = pairs[k];
    const float s = pt.view(views[pr.view], pr, h, j, i, taps);
    if (s > best) {
      best = s;
      best_view = k + 1;
    }
  }
  return best;
}

}  // namespace dn
