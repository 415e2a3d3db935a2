// Device-side steps of DepthmapCleaner::Clean and DepthmapPruner::Prune
// (reference opensfm/src/lib/dense/src/depthmap.cc:524-555 and :577-637),
// shared by the single-map kernels, the batched kernels (cleanprune.cu) and
// the persistent PatchMatch launch (kernels.cu).
//
// The keep/drop decisions compare depths against a relative threshold, so a
// last-bit difference in the projected depth can flip a pixel.  The
// geometry therefore follows the reference's own evaluation order in double
// (round-to-nearest intrinsics, no contraction) and rounds to float exactly
// where the reference stores a cv::Vec3f, which makes the masks and point
// lists bit-identical to the reference's.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace dn {

__device__ inline void m3v_rn(const double* a, const double x[3], double y[3]) {
#pragma unroll
  for (int r = 0; r < 3; ++r) y[r] = dot3_rn(a + 3 * r, x[0], x[1], x[2]);
}
__device__ inline void m3tv_rn(const double* a, const double x[3], double y[3]) {
#pragma unroll
  for (int r = 0; r < 3; ++r)
    y[r] = __dadd_rn(__dadd_rn(__dmul_rn(a[r], x[0]), __dmul_rn(a[3 + r], x[1])),
                     __dmul_rn(a[6 + r], x[2]));
}

// Backproject (depthmap.cc:108-112): R^T ((depth K^-1) q - t), rounded to
// float as the reference's cv::Vec3f result.
__device__ inline void backproject_f(double x, double y, double depth, const double* Kinv,
                                     const double* R, const double* t, float out[3]) {
  double M[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) M[k] = __dmul_rn(Kinv[k], depth);
  double p[3];
  p[0] = __dsub_rn(dot3_rn(M, x, y, 1.0), t[0]);
  p[1] = __dsub_rn(dot3_rn(M + 3, x, y, 1.0), t[1]);
  p[2] = __dsub_rn(dot3_rn(M + 6, x, y, 1.0), t[2]);
  double X[3];
  m3tv_rn(R, p, X);
  out[0] = (float)X[0];
  out[1] = (float)X[1];
  out[2] = (float)X[2];
}

// Project (depthmap.cc:104-106): K (R X + t) in double.
__device__ inline void project_d(const float Xf[3], const double* K, const double* R,
                                 const double* t, double out[3]) {
  const double X[3] = {Xf[0], Xf[1], Xf[2]};
  double p[3];
  m3v_rn(R, X, p);
#pragma unroll
  for (int k = 0; k < 3; ++k) p[k] = __dadd_rn(p[k], t[k]);
  m3v_rn(K, p, out);
}

// LinearInterpolation<float> (depthmap.cc:14-30) in the reference's float order.
__device__ inline float bilinear_f32(const float* im, int W, int H, int stride, float y, float x) {
  if (x < 0.0f || x >= (float)(W - 1) || y < 0.0f || y >= (float)(H - 1)) return 0.0f;
  const int ix = (int)x, iy = (int)y;
  const float dx = __fsub_rn(x, (float)ix), dy = __fsub_rn(y, (float)iy);
  const float* r0 = im + (size_t)iy * stride + ix;
  const float* r1 = r0 + stride;
  const float i00 = __ldg(r0), i01 = __ldg(r0 + 1), i10 = __ldg(r1), i11 = __ldg(r1 + 1);
  const float a = __fsub_rn(1.0f, dx);
  const float i0 = __fadd_rn(__fmul_rn(a, i00), __fmul_rn(dx, i01));
  const float i1 = __fadd_rn(__fmul_rn(a, i10), __fmul_rn(dx, i11));
  return __fadd_rn(__fmul_rn(__fsub_rn(1.0f, dy), i0), __fmul_rn(dy, i1));
}

// K^-1 with the cofactor form scaled by 1/det (cv::Matx33d::inv).
__device__ inline void inv3_rn(const double* a, double* r) {
  auto A = [&](int i, int j) { return a[3 * i + j]; };
  auto cof = [&](double p, double q, double s, double u) {
    return __dsub_rn(__dmul_rn(p, q), __dmul_rn(s, u));
  };
  double d = __dadd_rn(__dsub_rn(__dmul_rn(A(0, 0), cof(A(1, 1), A(2, 2), A(2, 1), A(1, 2))),
                                 __dmul_rn(A(0, 1), cof(A(1, 0), A(2, 2), A(2, 0), A(1, 2)))),
                       __dmul_rn(A(0, 2), cof(A(1, 0), A(2, 1), A(2, 0), A(1, 1))));
  if (d == 0.0) {
#pragma unroll
    for (int k = 0; k < 9; ++k) r[k] = 0.0;
    return;
  }
  d = __ddiv_rn(1.0, d);
  r[0] = __dmul_rn(cof(A(1, 1), A(2, 2), A(1, 2), A(2, 1)), d);
  r[1] = __dmul_rn(cof(A(0, 2), A(2, 1), A(0, 1), A(2, 2)), d);
  r[2] = __dmul_rn(cof(A(0, 1), A(1, 2), A(0, 2), A(1, 1)), d);
  r[3] = __dmul_rn(cof(A(1, 2), A(2, 0), A(1, 0), A(2, 2)), d);
  r[4] = __dmul_rn(cof(A(0, 0), A(2, 2), A(0, 2), A(2, 0)), d);
  r[5] = __dmul_rn(cof(A(0, 2), A(1, 0), A(0, 0), A(1, 2)), d);
  r[6] = __dmul_rn(cof(A(1, 0), A(2, 1), A(1, 1), A(2, 0)), d);
  r[7] = __dmul_rn(cof(A(0, 1), A(2, 0), A(0, 0), A(2, 1)), d);
  r[8] = __dmul_rn(cof(A(0, 0), A(1, 1), A(0, 1), A(1, 0)), d);
}

// ----------------------------------------------------------------------
// Cleaner: a pixel keeps its depth if at least min_views views (itself
// included) see a depth within thr * z of the reprojected point's depth.

// One pixel of DepthmapCleaner::Clean for the reference view rv (K^-1 in
// Kinv) against the views others[0..n): the value the cleaned map keeps.
__device__ inline float clean_pixel(const CleanView* __restrict__ views, const CleanView& rv,
                                    const double* Kinv, const int* __restrict__ others,
                                    int n_others, int i, int j, float thr, int min_views) {
  const float depth = rv.depth[(size_t)i * rv.stride + j];
  int consistent = 1;
  // A zero depth is dropped whatever the count (the kept value is 0), so
  // only the general case pays for the projections.
  if (depth != 0.0f) {
    float X[3];
    backproject_f((double)j, (double)i, (double)depth, Kinv, rv.R, rv.t, X);
    for (int k = 0; k < n_others; ++k) {
      const CleanView& ov = views[others[k]];
      double rp[3];
      project_d(X, ov.K, ov.R, ov.t, rp);
      const float r0 = (float)rp[0], r1 = (float)rp[1], r2 = (float)rp[2];
      if ((double)r2 < 1e-8 || isnan(r2)) continue;
      const float u = __fdiv_rn(r0, r2), v = __fdiv_rn(r1, r2);
      const float dr = bilinear_f32(ov.depth, ov.W, ov.H, ov.stride, v, u);
      if (fabsf(__fsub_rn(dr, r2)) < __fmul_rn(r2, thr)) consistent++;
    }
  }
  return (consistent >= min_views) ? depth : 0.0f;
}

// Every map of a batch in one launch: tile (map, tx, ty) covers the
// blockDim.x x blockDim.y pixels at (tx bx, ty by) of that map.
__device__ inline void clean_tile(const CleanView* __restrict__ views,
                                  const CleanMap* __restrict__ cmaps,
                                  const int* __restrict__ lists, int4 tl, float thr,
                                  int min_views) {
  __shared__ double Kinv[9];
  const CleanMap& cm = cmaps[tl.x];
  const CleanView& rv = views[tl.x];
  __syncthreads();  // Kinv of the previous tile (persistent blocks) is no longer read
  if (threadIdx.x == 0 && threadIdx.y == 0) inv3_rn(rv.K, Kinv);
  __syncthreads();
  const int j = tl.y * blockDim.x + threadIdx.x, i = tl.z * blockDim.y + threadIdx.y;
  if (i >= rv.H || j >= rv.W) return;
  cm.out[(size_t)i * rv.W + j] =
      clean_pixel(views, rv, Kinv, lists + cm.list_off, cm.n, i, j, thr, min_views);
}

// ----------------------------------------------------------------------
// Pruner.

// cv::normalize(Vec3f): multiply by 1 / ||v|| (norm in double).
__device__ inline void normalize3f(const float* v, float out[3]) {
  const double x = v[0], y = v[1], z = v[2];
  const double s = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
  const double nv = __dsqrt_rn(s);
  const double a = nv != 0.0 ? __ddiv_rn(1.0, nv) : 0.0;
  out[0] = (float)__dmul_rn(x, a);
  out[1] = (float)__dmul_rn(y, a);
  out[2] = (float)__dmul_rn(z, a);
}

constexpr int kPruneBlock = 256;

__device__ inline long long to_int64_x86(double x) {
  if (isnan(x) || x >= 9223372036854775808.0 || x < -9223372036854775808.0)
    return (long long)0x8000000000000000ull;
  return (long long)x;
}

// Decision of one pixel; on keep, also the outputs (point, R^T n).
// R1_normal = (float)R^T * n in float (cv::Matx33f * cv::Vec3f).
__device__ inline void world_normal(const PruneView& rv, const float nrm[3], float out[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float s = 0.0f;
#pragma unroll
    for (int b = 0; b < 3; ++b) s = __fadd_rn(s, __fmul_rn((float)rv.R[3 * b + a], nrm[b]));
    out[a] = s;
  }
}

__device__ inline bool prune_pixel(const PruneView* __restrict__ views, int n_views,
                                   const double* Kinv, int i, int j, float thr, float pt[3],
                                   float nrm_out[3]) {
  const PruneView& rv = views[0];
  const size_t pix = (size_t)i * rv.W + j;
  const float depth = rv.depth[pix];
  if (depth <= 0.0f) return false;
  float nrm[3];
  normalize3f(rv.plane + (size_t)rv.plane_stride * pix, nrm);
  const float area = (float)__dmul_rn((double)__fdiv_rn(-nrm[2], depth), rv.K[0]);
  backproject_f((double)j, (double)i, (double)depth, Kinv, rv.R, rv.t, pt);
  for (int o = 1; o < n_views; ++o) {
    const PruneView& ov = views[o];
    double rp[3];
    project_d(pt, ov.K, ov.R, ov.t, rp);
    if (rp[2] < 1e-8 || isnan(rp[2])) continue;
    const double fu = __dadd_rn(__ddiv_rn(rp[0], rp[2]), 0.5);
    const double fv = __dadd_rn(__ddiv_rn(rp[1], rp[2]), 0.5);
    // static_cast<int64_t> then narrowing to int (IsInsideImage takes
    // ints), with x86-64's result for NaN / out-of-range doubles (INT64_MIN).
    const int iu = (int)to_int64_x86(fu), iv = (int)to_int64_x86(fv);
    if (!(iv >= 0 && iv < ov.H && iu >= 0 && iu < ov.W)) continue;
    const size_t q = (size_t)iv * ov.W + iu;
    const float dr = ov.depth[q];
    const float keepf = __fsub_rn(1.0f, thr);
    if ((double)dr > __dmul_rn((double)keepf, rp[2])) {
      float no[3];
      normalize3f(ov.plane + (size_t)ov.plane_stride * q, no);
      if (dr == 0.0f || __dmul_rn((double)__fdiv_rn(-no[2], dr), ov.K[0]) > (double)area)
        return false;
    }
  }
  world_normal(rv, nrm, nrm_out);
  return true;
}

// The point and world normal of a kept pixel, as prune_pixel computes them
// (the same operations, without the checks against the other views).
__device__ inline void prune_point(const PruneView* __restrict__ views, const double* Kinv, int i,
                                   int j, float pt[3], float nrm_out[3]) {
  const PruneView& rv = views[0];
  const size_t pix = (size_t)i * rv.W + j;
  float nrm[3];
  normalize3f(rv.plane + (size_t)rv.plane_stride * pix, nrm);
  backproject_f((double)j, (double)i, (double)rv.depth[pix], Kinv, rv.R, rv.t, pt);
  world_normal(rv, nrm, nrm_out);
}

// Block-level steps of the pruner, for any block of B threads (a multiple
// of 32, 1-D or 2-D, warps along x): B consecutive pixels per block.
template <int B>
__device__ inline void prune_flags_block(const PruneView* __restrict__ views, int n_views,
                                         float thr, uint8_t* __restrict__ keep,
                                         uint32_t* __restrict__ block_counts, int block) {
  __shared__ double Kinv[9];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  __syncthreads();  // Kinv of a previous block (persistent blocks) is no longer read
  if (tid == 0) inv3_rn(views[0].K, Kinv);
  __syncthreads();
  const int W = views[0].W, H = views[0].H;
  const long k = (long)block * B + tid;
  bool kp = false;
  if (k < (long)W * H) {
    const int i = (int)(k / W), j = (int)(k - (long)i * W);
    float pt[3], nr[3];
    kp = prune_pixel(views, n_views, Kinv, i, j, thr, pt, nr);
    keep[k] = kp ? 1 : 0;
  }
  const int c = __syncthreads_count(kp);
  if (tid == 0) block_counts[block] = (uint32_t)c;
}

// Exclusive scan of n block counts by one block of any size (a multiple of
// 32, at most 1024 threads); the total in offsets[n] and *total.
__device__ inline void scan_counts_block(const uint32_t* __restrict__ counts, int n,
                                         uint32_t* __restrict__ offsets,
                                         unsigned long long* total) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry;
  const int nt = blockDim.x * blockDim.y, tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nw = nt / 32, lane = tid & 31, warp = tid >> 5;
  __syncthreads();
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += nt) {
    const int idx = base + tid;
    const uint32_t v = idx < n ? counts[idx] : 0;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t sm = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, sm, o);
        if (lane >= o) sm += y;
      }
      if (lane < nw) warp_sums[lane] = sm;
    }
    __syncthreads();
    const uint32_t before = (warp ? warp_sums[warp - 1] : 0) + carry;
    if (idx < n) offsets[idx] = before + x - v;
    __syncthreads();
    if (tid == nt - 1) carry = before + x;
    __syncthreads();
  }
  if (tid == 0) {
    offsets[n] = carry;
    if (total) *total = carry;
  }
}

// The kept pixels' points, normals, colours and labels at their offsets
// (the flags are final: the views and the threshold only name the pruner).
template <int B>
__device__ inline void prune_write_block(const PruneView* __restrict__ views, int /*n_views*/,
                                         float /*thr*/, const uint8_t* __restrict__ keep,
                                         const uint32_t* __restrict__ offsets, PruneOut out,
                                         int block) {
  __shared__ double Kinv[9];
  __shared__ uint32_t warp_base[B / 32];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  __syncthreads();  // shared state of a previous block is no longer read
  if (tid == 0) inv3_rn(views[0].K, Kinv);
  const int W = views[0].W, H = views[0].H;
  const long k = (long)block * B + tid;
  const bool kp = k < (long)W * H && keep[k];
  const int lane = tid & 31, warp = tid >> 5;
  const uint32_t ballot = __ballot_sync(0xffffffffu, kp);
  if (lane == 0) warp_base[warp] = __popc(ballot);
  __syncthreads();
  if (tid == 0) {
    uint32_t sm = offsets[block];
    for (int w = 0; w < B / 32; ++w) {
      const uint32_t c = warp_base[w];
      warp_base[w] = sm;
      sm += c;
    }
  }
  __syncthreads();
  if (!kp) return;
  const uint32_t pos = warp_base[warp] + __popc(ballot & ((1u << lane) - 1u));
  const int i = (int)(k / W), j = (int)(k - (long)i * W);
  float pt[3], nr[3];
  prune_point(views, Kinv, i, j, pt, nr);
  const PruneView& rv = views[0];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    out.points[3 * (size_t)pos + a] = pt[a];
    out.normals[3 * (size_t)pos + a] = nr[a];
    out.colors[3 * (size_t)pos + a] = rv.color ? rv.color[3 * k + a] : rv.gray[k];
  }
  out.labels[pos] = rv.label ? rv.label[k] : 0;
}

}  // namespace dn
