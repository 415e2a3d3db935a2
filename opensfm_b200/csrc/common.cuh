// Device-side data layout and helpers shared by the dense kernels.
//
// HBM layout (one reconstruction = a set of views + a set of depthmaps):
//   ViewDev  per view:  FP16 image [H][W] (uint8 intensities are exact in
//            FP16), optional uint8 mask, and a bilinear coefficient table
//            `quad` [(H-1+2P)][TP] of 4 x FP16 (8 bytes; the coefficients
//            are integers of magnitude <= 510, exact in FP16; see
//            build_quad_kernel).
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

// Coefficient table rows have a pitch TP = 1024 k - 1 entries (k a power of
// two).  With the floor trick t = x + M rounded down, M = 2^23 + 2^22 / k,
// the 32-bit product bits(ty) * TP + bits(tx) equals iy * TP + ix exactly
// (mod 2^32), so one IMAD turns the two biased floats into the entry index.
struct ViewDev {
  const __half* img;     // [H][W]
  const uint8_t* mask;   // [H][W] or null (all valid)
  const uint2* quad;     // [TH][TP] x 4 FP16, entry (ix, iy) at (iy + P) * TP + ix + P
  const uint2* quad0;    // &quad[entry (0, 0)]
  int W, H, TP, TH;
  float cbias;           // intensity centring constant folded into quad.x
  float magic;           // M for this pitch
  int pad_[2];
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
  uint8_t* changed;                        // [H][W] active-pixel flags (kMoved | kValid)
  float* prop_init;                        // [H][W][3] learned proposal planes
  long long prop_off;                      // first point of the map in the proposal grid
  int prop_W, prop_H;                      // proposal grid (W, H divided by the stride)
  int prop_S;                              // the map's proposal-grid stride
  // Active-pixel lists (list-mode half-passes): the pixels (y W + x) of
  // the half-pass's colour that are updated, and their number.
  int* alist;                              // [H W] capacity
  int* acount;                             // one counter
  int hp_tile0, hp_tiles;                  // the map's range in the half-pass tile list
};

// Active-pixel flags (MapDev::changed): kValid is set by the initialisation
// on every pixel it gives a plane (the pixels the half-passes update; it
// never changes after), kMoved by an update whose depth moved.
constexpr uint8_t kMoved = 1, kValid = 2;

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
  int variant;               // lanes per pixel (init and half-passes)
  // PatchMatch candidate schedule (defaults follow PatchMatchUpdatePixel,
  // depthmap.cc:305-374): adjacent planes, far planes, refinements and the
  // first refinement's depth / normal-slope ranges.
  int use_near, use_far, n_refine;
  float depth_range0, normal_range0;
  int use_knight;  // the 8 knight-move pixels (+-1, +-2), (+-2, +-1) as candidates
  // Active pixels: from half-pass 2 on, a pixel is updated only if its own
  // depth or one of its 4 neighbours' depths moved at their last update
  // (MapDev::changed); otherwise its state is kept as it is.  A depth moves
  // when it changes by more than active_tol relative (active_tol = 0: any
  // change of the plane counts).
  int active;
  float active_tol;
  // Settled start (active pixels only): the initialisation marks a pixel
  // as moved only if its initial score is below seed_score, and the active
  // rule applies from half-pass active_from (2 by default: the first two
  // update every pixel; 0 with a settled start).
  float seed_score;
  int active_from;
  int learned;  // initialise from MapDev::prop_init instead of MapDev::init
  int init_fallback;  // given planes: keep the random plane where it scores higher
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

// Where a reference patch is read: src(dy, dx) is the intensity at offset
// (dy, dx) from the centre pixel.  TileSrc reads the block's float tile in
// shared memory (centre at tile row ly, column lx); ImgSrc reads the view's
// FP16 image in global memory (centre (i, j), inside the image).  Both give
// the same values: the tile holds the image converted to float.
struct TileSrc {
  const float* tile;
  int pitch, ly, lx;
  __device__ float operator()(int dy, int dx) const { return tile[(ly + dy) * pitch + lx + dx]; }
};
struct ImgSrc {
  const __half* img;
  int W, i, j;
  __device__ float operator()(int dy, int dx) const {
    return __half2float(img[(size_t)(i + dy) * W + (j + dx)]);
  }
};

// Builds the reference patch terms of a pixel from src.
template <int HPZ, class Src>
__device__ inline void ref_patch_build(RefPatch<HPZ>& rp, const Src& src) {
  const float c = src(0, 0);
  const float dcf = 1.0f / 5000.0f;  // 1 / (2 * 50^2)
  const float dxf = 1.0f / 50.0f;    // 1 / (2 * 5^2)
  float sw = 0.f, swx = 0.f;
  float xs[RefPatch<HPZ>::N];
#pragma unroll
  for (int dy = -HPZ; dy <= HPZ; ++dy)
#pragma unroll
    for (int dx = -HPZ; dx <= HPZ; ++dx) {
      const int t = (dy + HPZ) * (2 * HPZ + 1) + (dx + HPZ);
      const float x = src(dy, dx);
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
// From a float tile in shared memory (ly, lx: tile coordinates of the centre).
template <int HPZ>
__device__ inline void ref_patch_from_tile(RefPatch<HPZ>& rp, const float* tile, int pitch,
                                           int ly, int lx) {
  ref_patch_build<HPZ>(rp, TileSrc{tile, pitch, ly, lx});
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
// var_y = 0, NCC = -1), kFast (inside the padded table), kSlow (leaves the
// padded table: taps clamped), kDegenerate (w == 0: NCC = -1).
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
  const float rw = __frcp_rn(w);  // 1 / w, correctly rounded, without the divide's slow path
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
                    (wp.Y0 - ey >= lo) && (wp.Y0 + ey < Hm1 + (float)kPad - 0.01f);
  wp.mode = fast ? kFast : kSlow;
  return wp;
}

// One coefficient entry (e0, e1, e2, e3) as FP32 (exact: the FP16 values are
// small integers).
__device__ __forceinline__ float4 quad_entry(const uint2* base, int off) {
  const uint2 h = __ldg(base + off);
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&h.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&h.y));
  return make_float4(a.x, a.y, b.x, b.y);
}

// Bilinear sample at (x, y) inside the padded table: floor by adding the
// magic constant rounding down, exact fractions, one IMAD for the entry
// index, one 8-byte load and three FMAs:  y - cbias = e0 + fx e1 +
// fy (e2 + fx e3).
__device__ inline float table_sample(const ViewDev& vw, float x, float y) {
  const float M = vw.magic;
  const float tx = __fadd_rd(x, M), ty = __fadd_rd(y, M);
  const float fx = x - (tx - M), fy = y - (ty - M);
  const int off = (int)(__float_as_uint(ty) * (unsigned)vw.TP + __float_as_uint(tx));
  const float4 q = quad_entry(vw.quad0, off);
  return fmaf(fy, fmaf(fx, q.w, q.z), fmaf(fx, q.y, q.x));
}

// Same, clamped: taps outside the padded table read its corner entry, whose
// sample is the reference's zero.
__device__ inline float table_sample_clamped(const ViewDev& vw, float x, float y) {
  const float xlo = -(float)kPad, xhi = (float)(vw.W - 1 + kPad);
  const float ylo = -(float)kPad, yhi = (float)(vw.H - 1 + kPad);
  if (x >= xlo && x < xhi && y >= ylo && y < yhi) return table_sample(vw, x, y);
  return quad_entry(vw.quad, 0).x;
}

// Per-patch centring value for the y sums: the table sample at the floor
// of the patch centre (the texel value there minus cbias), or, when the
// patch leaves the padded table, the clamped sample at the centre.  Any
// finite shift leaves the NCC unchanged in exact arithmetic; one near the
// patch's own mean keeps var_y free of cancellation in FP32 even where the
// patch is far from the view's mean intensity (flat sky, bright walls).
template <bool CLAMP>
__device__ inline float patch_shift(const ViewDev& vw, const Warp& wp) {
  if (CLAMP) return table_sample_clamped(vw, wp.X0, wp.Y0);
  const float M = vw.magic;
  const float tx = __fadd_rd(wp.X0, M), ty = __fadd_rd(wp.Y0, M);
  const int off = (int)(__float_as_uint(ty) * (unsigned)vw.TP + __float_as_uint(tx));
  return quad_entry(vw.quad0, off).x;
}

template <int HPZ>
__device__ inline float ncc_finish(const RefPatch<HPZ>& rp, float s1, float s2, float s3) {
  const float my = s1 * rp.inv_sw;
  const float vary = fmaf(s2, rp.inv_sw, -my * my);
  if (rp.varx < 0.1f || vary < 0.1f) return -1.0f;
  return (s3 * rp.inv_sw) * rsqrtf(rp.varx * vary);
}

// Bilateral NCC of the reference patch against one matching view under
// hypothesis h (ComputePlaneImageScore, depthmap.cc:441-478; NCCEstimator,
// depthmap.cc:46-74).  Same local affine warp of the plane-induced
// homography, tap positions X0 + ax dx + bx dy in float as the reference
// forms them, same bilinear sample with zeros outside [0,W-1) x [0,H-1),
// same weights.  Sums are mean-centred: x by the patch's weighted mean
// (hoisted), y by a value near the patch's own mean (patch_shift).
template <int HPZ, bool CLAMP>
__device__ inline float ncc_walk(const RefPatch<HPZ>& rp, const ViewDev& vw, const Warp& wp) {
  const float sh = patch_shift<CLAMP>(vw, wp);
  float s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
  for (int dy = -HPZ; dy <= HPZ; ++dy) {
    const float xr = fmaf(wp.bx, (float)dy, wp.X0), yr = fmaf(wp.by, (float)dy, wp.Y0);
#pragma unroll
    for (int dx = -HPZ; dx <= HPZ; ++dx) {
      const float x = fmaf(wp.ax, (float)dx, xr), yv = fmaf(wp.ay, (float)dx, yr);
      const float y =
          (CLAMP ? table_sample_clamped(vw, x, yv) : table_sample(vw, x, yv)) - sh;
      const int t = (dy + HPZ) * (2 * HPZ + 1) + (dx + HPZ);
      const float wy = rp.w[t] * y;
      s1 += wy;
      s2 = fmaf(wy, y, s2);
      s3 = fmaf(rp.wx[t], y, s3);
    }
  }
  return ncc_finish<HPZ>(rp, s1, s2, s3);
}

template <int HPZ>
__device__ inline float ncc_view(const RefPatch<HPZ>& rp, const ViewDev& vw, const PairDev& pr,
                                 const Hyp& h, float j, float i, unsigned& taps) {
  const Warp wp = warp_setup<HPZ>(vw, pr, h, j, i);
  if (wp.mode == kOutside || wp.mode == kDegenerate) return -1.0f;
  taps += RefPatch<HPZ>::N;
  if (wp.mode == kSlow) return ncc_walk<HPZ, true>(rp, vw, wp);
  return ncc_walk<HPZ, false>(rp, vw, wp);
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
// Packed FP32 pairs: sm_100 executes add / sub / mul / fma on two FP32 values
// held in a 64-bit register pair with one instruction (.f32x2), each half
// rounded exactly as the scalar instruction rounds it.  The FP32 pipe does
// the same work, but the walk below issues about a third fewer instructions,
// which leaves issue slots for its loads and integer work.
typedef unsigned long long u64;
__device__ __forceinline__ u64 pk2(float a, float b) {
  u64 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float lo2(u64 r) {
  float a;
  asm("{\n\t.reg .f32 unused;\n\tmov.b64 {%0, unused}, %1;\n\t}" : "=f"(a) : "l"(r));
  return a;
}
__device__ __forceinline__ float hi2(u64 r) {
  float b;
  asm("{\n\t.reg .f32 unused;\n\tmov.b64 {unused, %0}, %1;\n\t}" : "=f"(b) : "l"(r));
  return b;
}
__device__ __forceinline__ u64 add2(u64 a, u64 b) {
  u64 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ u64 add2_rd(u64 a, u64 b) {
  u64 d;
  asm("add.rm.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ u64 sub2(u64 a, u64 b) {
  u64 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ u64 mul2(u64 a, u64 b) {
  u64 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c) {
  u64 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// FP16 halves of a 32-bit word as FP32 (exact), and the low half plus an
// FP32 value in one rounding: sm_100's mixed-precision add (.f32.f16).
__device__ __forceinline__ float h16lo(unsigned w) {
  float r;
  asm("{\n\t.reg .b16 l, h;\n\tmov.b32 {l, h}, %1;\n\tcvt.f32.f16 %0, l;\n\t}" : "=f"(r) : "r"(w));
  return r;
}
__device__ __forceinline__ float h16hi(unsigned w) {
  float r;
  asm("{\n\t.reg .b16 l, h;\n\tmov.b32 {l, h}, %1;\n\tcvt.f32.f16 %0, h;\n\t}" : "=f"(r) : "r"(w));
  return r;
}
__device__ __forceinline__ float h16lo_add(unsigned w, float c) {
  float r;
  asm("{\n\t.reg .b16 l, h;\n\tmov.b32 {l, h}, %1;\n\tadd.rn.f32.f16 %0, l, %2;\n\t}"
      : "=f"(r) : "r"(w), "f"(c));
  return r;
}

// ------------------------------------------------------------------------
// Cooperative 7 x 7 patch: L lanes (2, 4 or 8, adjacent in the warp) share
// one pixel, each lane holding the weights of its slots (coop_slot).  With 4
// or 8 lanes the patch is padded to 8 columns: lane l owns columns l, l + L,
// ... (8 / L columns x 7 rows), and the padding column carries weight 0 and
// samples column 6's position; lanes l and l + 1 read neighbouring table
// entries (with 8 lanes a group reads a whole patch row at once).  With 2
// lanes the 49 taps split 25 / 24 without a padding column: each lane holds
// 25 slots (24 on lane 1, plus one of weight 0) instead of 28, in 12 pairs
// and one single.  The warp setup of a view is computed by one lane of the
// group and broadcast; the three sums are combined with XOR shuffles, so
// every lane of a group ends with the same score.
template <int L>
struct CoopPatch {
  static constexpr int C = 8 / L;  // columns per lane (4 and 8 lanes)
  static constexpr int S = L == 2 ? 25 : 7 * C;  // slots per lane
  static constexpr int P = S / 2;  // slot pairs per lane: slots 2k, 2k + 1
  static constexpr bool ODD = (S & 1) != 0;  // one column (L = 8): slot 6 alone
  u64 w2[P];                       // bilateral weights, packed in slot pairs
  u64 wx2[P];                      // w * (x - mean_x), packed likewise
  float wt, wxt;                   // the unpaired slot (ODD only)
  float inv_sw;
  float varx;
  int lane;
  unsigned mask;  // the lane group's bits in the warp
  int src0;       // warp lane of the group's lane 0
};

// Patch position (dx, dy in 0..6) of slot t of a lane; false for a padding
// slot (weight 0, sampled at a real position).  2 lanes: slots 0-13 are rows
// 0-6 of columns lane and lane + 2 (paired across the two columns), 14-19
// rows 0-5 of column lane + 4 (paired across rows), 20-23 rows 0-3 (lane 0)
// or 4-6 and a padding slot at row 6 (lane 1) of column 6, and 24 row 6 of
// column lane + 4.  4 and 8 lanes: slot r C + q is row r of column
// lane + L q, column 7 padding at column 6.
template <int L>
__host__ __device__ __forceinline__ bool coop_slot(int lane, int t, int& dx, int& dy) {
  if constexpr (L == 2) {
    if (t < 14) {
      dx = lane + 2 * (t & 1);
      dy = t >> 1;
    } else if (t < 20) {
      dx = lane + 4;
      dy = t - 14;
    } else if (t < 24) {
      dx = 6;
      dy = 4 * lane + (t - 20);
      if (dy > 6) {
        dy = 6;
        return false;
      }
    } else {
      dx = lane + 4;
      dy = 6;
    }
    return true;
  } else {
    constexpr int C = 8 / L;
    dx = lane + L * (t % C);
    dy = t / C;
    if (dx > 6) {
      dx = 6;
      return false;
    }
    return true;
  }
}

template <int L>
__device__ inline float group_sum(float v, unsigned mask) {
#pragma unroll
  for (int o = 1; o < L; o <<= 1) v += __shfl_xor_sync(mask, v, o);
  return v;
}

template <int L, class Src>
__device__ inline void coop_patch_build(CoopPatch<L>& cp, const Src& src, int lane, unsigned mask) {
  cp.lane = lane;
  cp.mask = mask;
  cp.src0 = (threadIdx.x & 31) - lane;
  const float c = src(0, 0);
  const float dcf = 1.0f / 5000.0f;
  const float dxf = 1.0f / 50.0f;
  float sw = 0.f, swx = 0.f;
  float ws[CoopPatch<L>::S], xs[CoopPatch<L>::S];
#pragma unroll
  for (int t = 0; t < CoopPatch<L>::S; ++t) {
    int dx, dy;
    const bool real = coop_slot<L>(lane, t, dx, dy);
    const float x = src(dy - 3, dx - 3);
    const float d = __fsub_rn(x, c);
    const int ddx = dx - 3, ddy = dy - 3;
    const float arg = __fsub_rn(__fmul_rn(__fmul_rn(-d, d), dcf),
                                __fmul_rn((float)(ddx * ddx + ddy * ddy), dxf));
    const float w = real ? expf(arg) : 0.0f;
    ws[t] = w;
    xs[t] = x;
    sw += w;
    swx = fmaf(w, x, swx);
  }
  sw = group_sum<L>(sw, mask);
  swx = group_sum<L>(swx, mask);
  const float inv_sw = 1.0f / sw;
  const float mx = swx * inv_sw;
  float sxx = 0.f;
  float wxs[CoopPatch<L>::S];
#pragma unroll
  for (int t = 0; t < CoopPatch<L>::S; ++t) {
    const float xc = xs[t] - mx;
    wxs[t] = ws[t] * xc;
    sxx = fmaf(wxs[t], xc, sxx);
  }
#pragma unroll
  for (int k = 0; k < CoopPatch<L>::P; ++k) {
    cp.w2[k] = pk2(ws[2 * k], ws[2 * k + 1]);
    cp.wx2[k] = pk2(wxs[2 * k], wxs[2 * k + 1]);
  }
  if (CoopPatch<L>::ODD) {
    cp.wt = ws[CoopPatch<L>::S - 1];
    cp.wxt = wxs[CoopPatch<L>::S - 1];
  } else {
    cp.wt = cp.wxt = 0.f;
  }
  sxx = group_sum<L>(sxx, mask);
  cp.inv_sw = inv_sw;
  cp.varx = sxx * inv_sw;
}
template <int L>
__device__ inline void coop_patch_from_tile(CoopPatch<L>& cp, const float* tile, int pitch, int ly,
                                            int lx, int lane, unsigned mask) {
  coop_patch_build<L>(cp, TileSrc{tile, pitch, ly, lx}, lane, mask);
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

// Column offset (relative to the lane's first column) of the lane's q-th
// column; the padding column (dx = 7, on lane L - 1) samples dx = 6.
template <int L>
__device__ inline float coop_col(int lane, int q) {
  constexpr int C = CoopPatch<L>::C;
  return (q == C - 1 && lane == L - 1) ? (float)(L * q - 1) : (float)(L * q);
}

// One lane's share of a view's walk, from the group's warp setup: taps
// clamped to the padded table (kSlow), one sample at a time.
template <int L>
__device__ inline float coop_walk_clamped(const CoopPatch<L>& cp, const ViewDev& vw,
                                          const Warp& wp) {
  if constexpr (L == 2) {
    // The slots in order, each at X0 + ax (dx - 3) + bx (dy - 3).
    const float sh = patch_shift<true>(vw, wp);
    float s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
    for (int t = 0; t < CoopPatch<L>::S; ++t) {
      int dx, dy;
      coop_slot<L>(cp.lane, t, dx, dy);
      const float fx = (float)(dx - 3), fy = (float)(dy - 3);
      const float x = fmaf(wp.ax, fx, fmaf(wp.bx, fy, wp.X0));
      const float yv = fmaf(wp.ay, fx, fmaf(wp.by, fy, wp.Y0));
      const float y = table_sample_clamped(vw, x, yv) - sh;
      float w, wx;
      if (t == CoopPatch<L>::S - 1) {
        w = cp.wt;
        wx = cp.wxt;
      } else {
        const u64 wpair = cp.w2[t >> 1], wxpair = cp.wx2[t >> 1];
        w = (t & 1) ? hi2(wpair) : lo2(wpair);
        wx = (t & 1) ? hi2(wxpair) : lo2(wxpair);
      }
      const float wy = w * y;
      s1 += wy;
      s2 = fmaf(wy, y, s2);
      s3 = fmaf(wx, y, s3);
    }
    return coop_finish<L>(cp, s1, s2, s3);
  } else {
    constexpr int C = CoopPatch<L>::C;
    const float dx0 = (float)(cp.lane - 3);
    const float xl = fmaf(wp.ax, dx0, fmaf(wp.bx, -3.0f, wp.X0));
    const float yl = fmaf(wp.ay, dx0, fmaf(wp.by, -3.0f, wp.Y0));
    const float sh = patch_shift<true>(vw, wp);
    float s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
    for (int r = 0; r < 7; ++r) {
      const float xr = fmaf(wp.bx, (float)r, xl), yr = fmaf(wp.by, (float)r, yl);
#pragma unroll
      for (int q = 0; q < C; ++q) {
        const float cq = coop_col<L>(cp.lane, q);
        const float x = fmaf(wp.ax, cq, xr), yv = fmaf(wp.ay, cq, yr);
        const float y = table_sample_clamped(vw, x, yv) - sh;
        const int t = r * C + q;
        float w, wx;
        if (CoopPatch<L>::ODD && t == CoopPatch<L>::S - 1) {
          w = cp.wt;
          wx = cp.wxt;
        } else {
          const u64 wpair = cp.w2[t >> 1], wxpair = cp.wx2[t >> 1];
          w = (t & 1) ? hi2(wpair) : lo2(wpair);
          wx = (t & 1) ? hi2(wxpair) : lo2(wxpair);
        }
        const float wy = w * y;
        s1 += wy;
        s2 = fmaf(wy, y, s2);
        s3 = fmaf(wx, y, s3);
      }
    }
    return coop_finish<L>(cp, s1, s2, s3);
  }
}

// Two table samples at the packed positions (X, Y), centred by nsh (minus
// the patch shift): returns the packed (sample - shift) values,
//   (e0 - shift) + fx e1 + fy (e2 + fx e3),
// with e0 - shift formed by the mixed-precision add while e0 is converted
// (exact when the shift is itself a table value) and the polynomial on
// packed pairs.
__device__ __forceinline__ u64 sample_pair(u64 X, u64 Y, u64 MM, unsigned TP,
                                           const uint2* __restrict__ q0, float nsh) {
  const u64 TX = add2_rd(X, MM), TY = add2_rd(Y, MM);
  const u64 FX = sub2(X, sub2(TX, MM)), FY = sub2(Y, sub2(TY, MM));
  // The index wraps modulo 2^32 by design: q0 is biased so that the
  // offset, read as a signed int, lands inside the table.
  const int oa = (int)(__float_as_uint(lo2(TY)) * TP + __float_as_uint(lo2(TX)));
  const int ob = (int)(__float_as_uint(hi2(TY)) * TP + __float_as_uint(hi2(TX)));
  const uint2 ha = __ldg(q0 + oa), hb = __ldg(q0 + ob);
  const u64 E0 = pk2(h16lo_add(ha.x, nsh), h16lo_add(hb.x, nsh));
  const u64 E1 = pk2(h16hi(ha.x), h16hi(hb.x));
  const u64 E2 = pk2(h16lo(ha.y), h16lo(hb.y));
  const u64 E3 = pk2(h16hi(ha.y), h16hi(hb.y));
  return fma2(FY, fma2(FX, E3, E2), fma2(FX, E1, E0));
}

// The same walk inside the padded table (kFast), two slots per step on
// packed FP32 pairs: tap positions, the floor (add rounding down to the
// magic constant), the fractions, the bilinear polynomial and the three
// weighted sums all run as .f32x2; the entry index stays scalar.  With
// 2 or 4 lanes a pair is two columns of one row; with 8 lanes (one column
// per lane) it is two rows, and row 6 is sampled alone.
template <int L>
__device__ inline float coop_walk_fast(const CoopPatch<L>& cp, const ViewDev& vw,
                                       const Warp& wp) {
  constexpr int C = CoopPatch<L>::C;
  const float dx0 = (float)(cp.lane - 3);
  const float xl = fmaf(wp.ax, dx0, fmaf(wp.bx, -3.0f, wp.X0));
  const float yl = fmaf(wp.ay, dx0, fmaf(wp.by, -3.0f, wp.Y0));
  const u64 MM = pk2(vw.magic, vw.magic);
  const unsigned TP = (unsigned)vw.TP;
  const uint2* __restrict__ q0 = vw.quad0;
  const float nsh = -patch_shift<false>(vw, wp);
  u64 S1 = 0ull, S2 = 0ull, S3 = 0ull;  // (+0.0f, +0.0f) pairs
  float t1 = 0.f, t2 = 0.f, t3 = 0.f;   // the unpaired slot
  if constexpr (L == 2) {
    // Columns lane and lane + 2, one row per step (slots 0-13).
    const u64 BX = pk2(wp.bx, wp.bx), BY = pk2(wp.by, wp.by);
    u64 X = pk2(xl, fmaf(wp.ax, 2.0f, xl)), Y = pk2(yl, fmaf(wp.ay, 2.0f, yl));
#pragma unroll
    for (int r = 0; r < 7; ++r) {
      const u64 YY = sample_pair(X, Y, MM, TP, q0, nsh);
      const u64 WY = mul2(cp.w2[r], YY);
      S1 = add2(S1, WY);
      S2 = fma2(WY, YY, S2);
      S3 = fma2(cp.wx2[r], YY, S3);
      if (r < 6) {
        X = add2(X, BX);
        Y = add2(Y, BY);
      }
    }
    // Column lane + 4, two rows per step (slots 14-19); its row 6 is slot 24.
    const float xb = fmaf(wp.ax, 4.0f, xl), yb = fmaf(wp.ay, 4.0f, yl);
    const u64 BX2 = pk2(2.0f * wp.bx, 2.0f * wp.bx), BY2 = pk2(2.0f * wp.by, 2.0f * wp.by);
    X = pk2(xb, __fadd_rn(xb, wp.bx));
    Y = pk2(yb, __fadd_rn(yb, wp.by));
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const u64 YY = sample_pair(X, Y, MM, TP, q0, nsh);
      const u64 WY = mul2(cp.w2[7 + k], YY);
      S1 = add2(S1, WY);
      S2 = fma2(WY, YY, S2);
      S3 = fma2(cp.wx2[7 + k], YY, S3);
      if (k < 2) {
        X = add2(X, BX2);
        Y = add2(Y, BY2);
      }
    }
    // Column 6 (slots 20-23): rows 0-3 on lane 0; rows 4-6 and row 6 again
    // (weight 0) on lane 1.
    const float lf = (float)cp.lane;
    const float x6 = fmaf(wp.bx, 4.0f * lf, fmaf(wp.ax, 6.0f - lf, xl));
    const float y6 = fmaf(wp.by, 4.0f * lf, fmaf(wp.ay, 6.0f - lf, yl));
    const float last = cp.lane ? 2.0f : 3.0f;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      if (k == 0) {
        X = pk2(x6, __fadd_rn(x6, wp.bx));
        Y = pk2(y6, __fadd_rn(y6, wp.by));
      } else {
        X = pk2(fmaf(wp.bx, 2.0f, x6), fmaf(wp.bx, last, x6));
        Y = pk2(fmaf(wp.by, 2.0f, y6), fmaf(wp.by, last, y6));
      }
      const u64 YY = sample_pair(X, Y, MM, TP, q0, nsh);
      const u64 WY = mul2(cp.w2[10 + k], YY);
      S1 = add2(S1, WY);
      S2 = fma2(WY, YY, S2);
      S3 = fma2(cp.wx2[10 + k], YY, S3);
    }
    const float y24 = table_sample(vw, fmaf(wp.bx, 6.0f, xb), fmaf(wp.by, 6.0f, yb)) + nsh;
    const float wy = cp.wt * y24;
    t1 = wy;
    t2 = wy * y24;
    t3 = cp.wxt * y24;
  } else if constexpr (C == 1) {
    const float c0 = coop_col<L>(cp.lane, 0);
    const float xc = fmaf(wp.ax, c0, xl), yc = fmaf(wp.ay, c0, yl);
    u64 X = pk2(xc, __fadd_rn(xc, wp.bx)), Y = pk2(yc, __fadd_rn(yc, wp.by));
    const u64 BX = pk2(2.0f * wp.bx, 2.0f * wp.bx), BY = pk2(2.0f * wp.by, 2.0f * wp.by);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const u64 YY = sample_pair(X, Y, MM, TP, q0, nsh);
      const u64 WY = mul2(cp.w2[k], YY);
      S1 = add2(S1, WY);
      S2 = fma2(WY, YY, S2);
      S3 = fma2(cp.wx2[k], YY, S3);
      X = add2(X, BX);
      Y = add2(Y, BY);
    }
    const float y6 = table_sample(vw, fmaf(wp.bx, 6.0f, xc), fmaf(wp.by, 6.0f, yc)) + nsh;
    const float wy = cp.wt * y6;
    t1 = wy;
    t2 = wy * y6;
    t3 = cp.wxt * y6;
  } else {
    constexpr int NP = C / 2;  // column pairs per lane
    u64 X[NP], Y[NP];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      const float c0 = coop_col<L>(cp.lane, 2 * m), c1 = coop_col<L>(cp.lane, 2 * m + 1);
      X[m] = pk2(fmaf(wp.ax, c0, xl), fmaf(wp.ax, c1, xl));
      Y[m] = pk2(fmaf(wp.ay, c0, yl), fmaf(wp.ay, c1, yl));
    }
    const u64 BX = pk2(wp.bx, wp.bx), BY = pk2(wp.by, wp.by);
#pragma unroll
    for (int r = 0; r < 7; ++r) {
#pragma unroll
      for (int m = 0; m < NP; ++m) {
        const u64 YY = sample_pair(X[m], Y[m], MM, TP, q0, nsh);
        const int k = r * NP + m;
        const u64 WY = mul2(cp.w2[k], YY);
        S1 = add2(S1, WY);
        S2 = fma2(WY, YY, S2);
        S3 = fma2(cp.wx2[k], YY, S3);
        if (r < 6) {
          X[m] = add2(X[m], BX);
          Y[m] = add2(Y[m], BY);
        }
      }
    }
  }
  return coop_finish<L>(cp, lo2(S1) + hi2(S1) + t1, lo2(S2) + hi2(S2) + t2,
                        lo2(S3) + hi2(S3) + t3);
}

template <int L>
__device__ inline Warp bcast_warp(const Warp& w, unsigned mask, int src) {
  Warp o;
  o.X0 = __shfl_sync(mask, w.X0, src);
  o.Y0 = __shfl_sync(mask, w.Y0, src);
  o.ax = __shfl_sync(mask, w.ax, src);
  o.bx = __shfl_sync(mask, w.bx, src);
  o.ay = __shfl_sync(mask, w.ay, src);
  o.by = __shfl_sync(mask, w.by, src);
  o.mode = __shfl_sync(mask, w.mode, src);
  return o;
}

template <int L>
__device__ inline float coop_eval(const CoopPatch<L>& cp, const ViewDev& vw, const Warp& wp,
                                  unsigned& taps) {
  if (wp.mode == kOutside || wp.mode == kDegenerate) return -1.0f;
  if (cp.lane == 0) taps += 49;
  if (wp.mode == kSlow) return coop_walk_clamped<L>(cp, vw, wp);
  return coop_walk_fast<L>(cp, vw, wp);
}

// Single view (sample mode): every lane computes the same setup.
template <int L>
__device__ inline float coop_ncc_view(const CoopPatch<L>& cp, const ViewDev& vw,
                                      const PairDev& pr, const Hyp& h, float j, float i,
                                      unsigned& taps) {
  const Warp wp = warp_setup<3>(vw, pr, h, j, i);
  return coop_eval<L>(cp, vw, wp, taps);
}

// Max over views: lane l of the group sets up views l, l + L, ...; each
// setup is broadcast to the group before the shared walk.
template <int L>
__device__ inline float coop_max(const CoopPatch<L>& cp, const ViewDev* views,
                                 const PairDev* pairs, int n_pairs, const Hyp& h, float j,
                                 float i, int& best_view, unsigned& taps) {
  float best = -1.0f;
  best_view = 0;
  for (int k0 = 0; k0 < n_pairs; k0 += L) {
    const int mine = min(k0 + cp.lane, n_pairs - 1);
    const PairDev& prm = pairs[mine];
    const Warp own = warp_setup<3>(views[prm.view], prm, h, j, i);
    const int nv = min(L, n_pairs - k0);
    for (int v = 0; v < nv; ++v) {
      const Warp wp = bcast_warp<L>(own, cp.mask, cp.src0 + v);
      const ViewDev& vw = views[pairs[k0 + v].view];
      const float s = coop_eval<L>(cp, vw, wp, taps);
      if (s > best) {
        best = s;
        best_view = k0 + v + 1;
      }
    }
  }
  return best;
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
  template <class Src>
  __device__ void build_src(const Src& src, int, unsigned) {
    ref_patch_build<HPZ>(rp, src);
  }
  __device__ float view(const ViewDev& vw, const PairDev& pr, const Hyp& h, float j, float i,
                        unsigned& taps) const {
    return ncc_view<HPZ>(rp, vw, pr, h, j, i, taps);
  }
  __device__ float max(const ViewDev* views, const PairDev* pairs, int n, const Hyp& h, float j,
                       float i, int& best_view, unsigned& taps) const {
    return ncc_max<HPZ>(rp, views, pairs, n, h, j, i, best_view, taps);
  }
};

template <int L>
struct CoopIface {
  CoopPatch<L> cp;
  __device__ void build(const float* tile, int pitch, int ly, int lx, int lane, unsigned mask) {
    coop_patch_from_tile<L>(cp, tile, pitch, ly, lx, lane, mask);
  }
  template <class Src>
  __device__ void build_src(const Src& src, int lane, unsigned mask) {
    coop_patch_build<L>(cp, src, lane, mask);
  }
  __device__ float view(const ViewDev& vw, const PairDev& pr, const Hyp& h, float j, float i,
                        unsigned& taps) const {
    return coop_ncc_view<L>(cp, vw, pr, h, j, i, taps);
  }
  __device__ float max(const ViewDev* views, const PairDev* pairs, int n, const Hyp& h, float j,
                       float i, int& best_view, unsigned& taps) const {
    return coop_max<L>(cp, views, pairs, n, h, j, i, best_view, taps);
  }
};
template <>
struct Patch<3, 2> : CoopIface<2> {};
template <>
struct Patch<3, 4> : CoopIface<4> {};
template <>
struct Patch<3, 8> : CoopIface<8> {};

template <int HPZ, int L>
__device__ inline float patch_max(const Patch<HPZ, L>& pt, const ViewDev* views,
                                  const PairDev* pairs, int n_pairs, const Hyp& h, float j,
                                  float i, int& best_view, unsigned& taps) {
  return pt.max(views, pairs, n_pairs, h, j, i, best_view, taps);
}

// ----------------------------------------------------------------------
// The depthmap's matching-view records (pair factors and view tables),
// copied to shared memory at the start of a tile: every candidate's
// homography setup and walk reads them there instead of through L1.
// p[k].view indexes v.
struct PairViewSm {
  ViewDev v[kMaxNbr];
  PairDev p[kMaxNbr];
};

__device__ inline void stage_pairs(PairViewSm& s, const MapDev& m, const ViewDev* views,
                                   const PairDev* pairs) {
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  if (t < m.n_pairs) {
    PairDev pr = pairs[m.pair0 + t];
    s.v[t] = views[pr.view];
    pr.view = t;
    s.p[t] = pr;
  }
}

}  // namespace dn
