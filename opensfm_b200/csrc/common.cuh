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

// Bilateral NCC of the reference patch against one matching view under
// hypothesis h (ComputePlaneImageScore, depthmap.cc:441-478; NCCEstimator,
// depthmap.cc:46-74).  Same local affine warp of the plane-induced
// homography, same bilinear sample with zeros outside [0,W-1) x [0,H-1),
// same weights.  Sums are mean-centred: x by the patch's weighted mean
// (hoisted), y by the view's constant cbias (folded into the table).
//
// Fast path: tap coordinates in 9.23 fixed point relative to the floor of
// the patch centre; the fraction bits become the float 1 + f directly and
// the table holds the bilinear polynomial in (1 + fx, 1 + fy), so one
// 16-byte load and three FMAs give the sample.  Slow path (patch leaves the
// padded table or is stretched > 200 px): float coordinates, clamped.
template <int HPZ>
__device__ inline float ncc_view(const RefPatch<HPZ>& rp, const ViewDev& vw, const PairDev& pr,
                                 const Hyp& h, float j, float i, unsigned& taps) {
  const float gq0 = fmaf(pr.G[0], j, fmaf(pr.G[1], i, pr.G[2]));
  const float gq1 = fmaf(pr.G[3], j, fmaf(pr.G[4], i, pr.G[5]));
  const float gq2 = fmaf(pr.G[6], j, fmaf(pr.G[7], i, pr.G[8]));
  const float u = fmaf(pr.e[0], h.fq, gq0);
  const float v = fmaf(pr.e[1], h.fq, gq1);
  const float w = fmaf(pr.e[2], h.fq, gq2);
  if (w == 0.0f) return -1.0f;
  const float H00 = fmaf(pr.e[0], h.f0, pr.G[0]), H01 = fmaf(pr.e[0], h.f1, pr.G[1]);
  const float H10 = fmaf(pr.e[1], h.f0, pr.G[3]), H11 = fmaf(pr.e[1], h.f1, pr.G[4]);
  const float H20 = fmaf(pr.e[2], h.f0, pr.G[6]), H21 = fmaf(pr.e[2], h.f1, pr.G[7]);
  const float rw = 1.0f / w;
  const float X0 = u * rw, Y0 = v * rw;
  const float ax = (H00 - H20 * X0) * rw;  // d x2 / d dx
  const float bx = (H01 - H21 * X0) * rw;  // d x2 / d dy
  const float ay = (H10 - H20 * Y0) * rw;  // d y2 / d dx
  const float by = (H11 - H21 * Y0) * rw;  // d y2 / d dy
  const float ex = HPZ * (fabsf(ax) + fabsf(bx));
  const float ey = HPZ * (fabsf(ay) + fabsf(by));
  const float Wm1 = (float)(vw.W - 1), Hm1 = (float)(vw.H - 1);
  // Every tap outside the image: all samples are 0, var_y = 0, NCC = -1.
  if (X0 + ex < -0.01f || X0 - ex >= Wm1 + 0.01f || Y0 + ey < -0.01f || Y0 - ey >= Hm1 + 0.01f)
    return -1.0f;
  float s1 = 0.f, s2 = 0.f, s3 = 0.f;
  const float lo = -(float)kPad + 0.01f;
  const bool fast = (X0 - ex >= lo) && (X0 + ex < Wm1 + (float)kPad - 0.01f) && (Y0 - ey >= lo) &&
                    (Y0 + ey < Hm1 + (float)kPad - 0.01f) && ex < 200.f && ey < 200.f;
  taps += RefPatch<HPZ>::N;
  if (fast) {
    const float fbx = floorf(X0), fby = floorf(Y0);
    const int ibx = (int)fbx, iby = (int)fby;
    const float sc = 8388608.0f;  // 2^23
    const int XS = __float2int_rn((X0 - fbx - HPZ * ax - HPZ * bx) * sc);
    const int YS = __float2int_rn((Y0 - fby - HPZ * ay - HPZ * by) * sc);
    const int AX = __float2int_rn(ax * sc), BX = __float2int_rn(bx * sc);
    const int AY = __float2int_rn(ay * sc), BY = __float2int_rn(by * sc);
    const float4* base = vw.quad + (size_t)(iby + kPad) * vw.TW + (ibx + kPad);
    const int TW = vw.TW;
#pragma unroll
    for (int dy = 0; dy <= 2 * HPZ; ++dy) {
      const int xr = XS + dy * BX, yr = YS + dy * BY;
#pragma unroll
      for (int dx = 0; dx <= 2 * HPZ; ++dx) {
        const int XF = xr + dx * AX, YF = yr + dx * AY;
        const int ix = XF >> 23, iy = YF >> 23;
        const float f1 = __int_as_float((XF & 0x7FFFFF) | 0x3F800000);
        const float g1 = __int_as_float((YF & 0x7FFFFF) | 0x3F800000);
        const float4 q = __ldg(base + iy * TW + ix);
        const float y = fmaf(g1, fmaf(f1, q.w, q.z), fmaf(f1, q.y, q.x));
        const int t = dy * (2 * HPZ + 1) + dx;
        const float wy = rp.w[t] * y;
        s1 += wy;
        s2 = fmaf(wy, y, s2);
        s3 = fmaf(rp.wx[t], y, s3);
      }
    }
  } else {
    const float xlo = -(float)kPad, xhi = Wm1 + (float)kPad;
    const float ylo = -(float)kPad, yhi = Hm1 + (float)kPad;
#pragma unroll
    for (int dy = -HPZ; dy <= HPZ; ++dy)
#pragma unroll
      for (int dx = -HPZ; dx <= HPZ; ++dx) {
        const float x = fmaf(bx, (float)dy, fmaf(ax, (float)dx, X0));
        const float yv = fmaf(by, (float)dy, fmaf(ay, (float)dx, Y0));
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
  }
  const float my = s1 * rp.inv_sw;
  const float vary = fmaf(s2, rp.inv_sw, -my * my);
  if (rp.varx < 0.1f || vary < 0.1f) return -1.0f;
  return (s3 * rp.inv_sw) * rsqrtf(rp.varx * vary);
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

}  // namespace dn
