// Cross-view consistency kernels: DepthmapCleaner::Clean and
// DepthmapPruner::Prune (reference opensfm/src/lib/dense/src/depthmap.cc
// :524-555 and :577-637).
//
// The keep/drop decisions compare depths against a relative threshold, so a
// last-bit difference in the projected depth can flip a pixel.  Both kernels
// therefore evaluate the geometry with the reference's own evaluation order
// in double (round-to-nearest intrinsics, no contraction) and round to float
// exactly where the reference stores a cv::Vec3f, which makes the masks and
// point lists bit-identical to the reference's.  The FP64 work per
// (pixel, view) is ~35 operations; both kernels are a few percent of a
// reconstruction's time.
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

__global__ void __launch_bounds__(256)
clean_kernel(const CleanView* __restrict__ views, int ref, const int* __restrict__ others,
             int n_others, int W, int H, float thr, int min_views, float* __restrict__ out) {
  __shared__ double Kinv[9];
  const CleanView& rv = views[ref];
  if (threadIdx.x == 0 && threadIdx.y == 0) inv3_rn(rv.K, Kinv);
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= H || j >= W) return;
  const float depth = rv.depth[(size_t)i * rv.stride + j];
  int consistent = 1;
  if (depth != 0.0f || min_views > 1) {
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
  }
  out[(size_t)i * W + j] = (consistent >= min_views) ? depth : 0.0f;
}

cudaError_t launch_clean(const CleanView* d_views, int ref, const int* d_others, int n_others,
                         int W, int H, float thr, int min_views, float* out, cudaStream_t s) {
  const dim3 blk(32, 8), grid((W + 31) / 32, (H + 7) / 8);
  clean_kernel<<<grid, blk, 0, s>>>(d_views, ref, d_others, n_others, W, H, thr, min_views, out);
  return cudaGetLastError();
}

// ----------------------------------------------------------------------
// GPUDepthmapCleaner::Clean (cleaner.cc:56-170; kernel acmmp_clean_depthmap,
// opencl_kernels.h:2155-2273).  Per pixel with depth > 0: back-project with
// the reference camera, project into each source; a source whose depth at
// that point is farther than (1 + carving) x the point's depth carves it;
// one within the relative threshold whose own point projects back within
// 2 px (L1) and the threshold of the reference depth counts as consistent.
// Keep if consistent (starting at 1) >= min_consistent and carved <
// max_carved.  All arithmetic is FP32 in the kernel's order with each
// operation rounded (no contraction); the source depth is sampled bilinearly
// with exact fractions (the reference asks the texture unit for a linear
// filter at the texel centre, the same interpolant).
struct Vec3f {
  float x, y, z;
};

// R^T p for row-major R (the kernel's camera-to-world rotation).
__device__ inline Vec3f rot_t(const float* R, float x, float y, float z) {
  return {__fadd_rn(__fadd_rn(__fmul_rn(R[0], x), __fmul_rn(R[3], y)), __fmul_rn(R[6], z)),
          __fadd_rn(__fadd_rn(__fmul_rn(R[1], x), __fmul_rn(R[4], y)), __fmul_rn(R[7], z)),
          __fadd_rn(__fadd_rn(__fmul_rn(R[2], x), __fmul_rn(R[5], y)), __fmul_rn(R[8], z))};
}
// R p + t.
__device__ inline Vec3f rot_add(const float* R, const float* t, Vec3f p) {
  return {__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(R[0], p.x), __fmul_rn(R[1], p.y)),
                              __fmul_rn(R[2], p.z)), t[0]),
          __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(R[3], p.x), __fmul_rn(R[4], p.y)),
                              __fmul_rn(R[5], p.z)), t[1]),
          __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(R[6], p.x), __fmul_rn(R[7], p.y)),
                              __fmul_rn(R[8], p.z)), t[2])};
}
// World point of pixel (u, v) at depth d: R^T ((u - cx) / fx * d - t, ...).
__device__ inline Vec3f backproject_px(const GpuCleanCam& c, float u, float v, float d) {
  const float cam_x = __fmul_rn(__fdiv_rn(__fsub_rn(u, c.K[2]), c.K[0]), d);
  const float cam_y = __fmul_rn(__fdiv_rn(__fsub_rn(v, c.K[5]), c.K[4]), d);
  return rot_t(c.R, __fsub_rn(cam_x, c.t[0]), __fsub_rn(cam_y, c.t[1]), __fsub_rn(d, c.t[2]));
}

__device__ inline float bilinear_exact(const float* d, int W, float u, float v) {
  const int ix = (int)u, iy = (int)v;  // u, v >= 0 here
  const float fx = __fsub_rn(u, (float)ix), fy = __fsub_rn(v, (float)iy);
  const float gx = __fsub_rn(1.0f, fx), gy = __fsub_rn(1.0f, fy);
  const float* p = d + (size_t)iy * W + ix;
  const float top = __fadd_rn(__fmul_rn(gx, p[0]), __fmul_rn(fx, p[1]));
  const float bot = __fadd_rn(__fmul_rn(gx, p[W]), __fmul_rn(fx, p[W + 1]));
  return __fadd_rn(__fmul_rn(gy, top), __fmul_rn(fy, bot));
}

__global__ void gpu_clean_kernel(const __grid_constant__ GpuCleanArgs a, float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= a.W || y >= a.H) return;
  const size_t idx = (size_t)y * a.W + x;
  const float d = a.ref[idx];
  if (!(d > 0.0f)) {
    out[idx] = 0.0f;
    return;
  }
  const GpuCleanCam& rc = a.cam[0];
  const Vec3f w = backproject_px(rc, (float)x, (float)y, d);
  int consistent = 1, carved = 0;
  for (int v = 0; v < a.n_src; ++v) {
    const GpuCleanCam& sc = a.cam[v + 1];
    const Vec3f s = rot_add(sc.R, sc.t, w);
    if (s.z <= 1e-6f) continue;
    const float su = __fadd_rn(__fdiv_rn(__fmul_rn(sc.K[0], s.x), s.z), sc.K[2]);
    const float sv = __fadd_rn(__fdiv_rn(__fmul_rn(sc.K[4], s.y), s.z), sc.K[5]);
    if (su < 0.0f || sv < 0.0f || su >= (float)(a.W - 1) || sv >= (float)(a.H - 1)) continue;
    const float sd = bilinear_exact(a.src[v], a.W, su, sv);
    if (!(sd > 0.0f)) continue;
    if (sd > __fmul_rn(s.z, __fadd_rn(1.0f, a.carving_threshold))) {
      ++carved;
      continue;
    }
    if (fabsf(__fsub_rn(sd, s.z)) >= __fmul_rn(s.z, a.same_depth_threshold)) continue;
    const Vec3f w2 = backproject_px(sc, su, sv, sd);
    const Vec3f r = rot_add(rc.R, rc.t, w2);
    if (r.z <= 1e-6f) continue;
    const float ru = __fadd_rn(__fdiv_rn(__fmul_rn(rc.K[0], r.x), r.z), rc.K[2]);
    const float rv = __fadd_rn(__fdiv_rn(__fmul_rn(rc.K[4], r.y), r.z), rc.K[5]);
    if (__fadd_rn(fabsf(__fsub_rn(ru, (float)x)), fabsf(__fsub_rn(rv, (float)y))) > 2.0f) continue;
    if (fabsf(__fsub_rn(r.z, d)) >= __fmul_rn(d, a.same_depth_threshold)) continue;
    ++consistent;
  }
  out[idx] = (consistent >= a.min_consistent && carved < a.max_carved) ? d : 0.0f;
}

cudaError_t launch_gpu_clean(const GpuCleanArgs& a, float* out, cudaStream_t s) {
  const dim3 blk(32, 8), grid((a.W + 31) / 32, (a.H + 7) / 8);
  gpu_clean_kernel<<<grid, blk, 0, s>>>(a, out);
  return cudaGetLastError();
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
  // R1_normal = (float)R^T * n in float (cv::Matx33f * cv::Vec3f).
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float s = 0.0f;
#pragma unroll
    for (int b = 0; b < 3; ++b) s = __fadd_rn(s, __fmul_rn((float)rv.R[3 * b + a], nrm[b]));
    nrm_out[a] = s;
  }
  return true;
}

__global__ void __launch_bounds__(kPruneBlock)
prune_flags_kernel(const PruneView* __restrict__ views, int n_views, float thr,
                   uint8_t* __restrict__ keep, uint32_t* __restrict__ block_counts) {
  __shared__ double Kinv[9];
  if (threadIdx.x == 0) inv3_rn(views[0].K, Kinv);
  __syncthreads();
  const int W = views[0].W, H = views[0].H;
  const long k = (long)blockIdx.x * kPruneBlock + threadIdx.x;
  bool kp = false;
  if (k < (long)W * H) {
    const int i = (int)(k / W), j = (int)(k - (long)i * W);
    float pt[3], nr[3];
    kp = prune_pixel(views, n_views, Kinv, i, j, thr, pt, nr);
    keep[k] = kp ? 1 : 0;
  }
  const int c = __syncthreads_count(kp);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = (uint32_t)c;
}

// Exclusive scan of the block counts in one block; total in offsets[n].
__global__ void __launch_bounds__(1024)
scan_counts_kernel(const uint32_t* __restrict__ counts, int n, uint32_t* __restrict__ offsets,
                   unsigned long long* total) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < n; base += 1024) {
    const int idx = base + threadIdx.x;
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
      uint32_t s = warp_sums[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      warp_sums[lane] = s;
    }
    __syncthreads();
    const uint32_t before = (warp ? warp_sums[warp - 1] : 0) + carry;
    if (idx < n) offsets[idx] = before + x - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry = before + x;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    offsets[n] = carry;
    if (total) *total = carry;
  }
}

__global__ void __launch_bounds__(kPruneBlock)
prune_write_kernel(const PruneView* __restrict__ views, int n_views, float thr,
                   const uint8_t* __restrict__ keep, const uint32_t* __restrict__ offsets,
                   PruneOut out) {
  __shared__ double Kinv[9];
  __shared__ uint32_t warp_base[kPruneBlock / 32];
  if (threadIdx.x == 0) inv3_rn(views[0].K, Kinv);
  const int W = views[0].W, H = views[0].H;
  const long k = (long)blockIdx.x * kPruneBlock + threadIdx.x;
  const bool kp = k < (long)W * H && keep[k];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t ballot = __ballot_sync(0xffffffffu, kp);
  if (lane == 0) warp_base[warp] = __popc(ballot);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = offsets[blockIdx.x];
    for (int w = 0; w < kPruneBlock / 32; ++w) {
      const uint32_t c = warp_base[w];
      warp_base[w] = s;
      s += c;
    }
  }
  __syncthreads();
  if (!kp) return;
  const uint32_t pos = warp_base[warp] + __popc(ballot & ((1u << lane) - 1u));
  const int i = (int)(k / W), j = (int)(k - (long)i * W);
  float pt[3], nr[3];
  prune_pixel(views, n_views, Kinv, i, j, thr, pt, nr);
  const PruneView& rv = views[0];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    out.points[3 * (size_t)pos + a] = pt[a];
    out.normals[3 * (size_t)pos + a] = nr[a];
    out.colors[3 * (size_t)pos + a] = rv.color ? rv.color[3 * k + a] : rv.gray[k];
  }
  out.labels[pos] = rv.label ? rv.label[k] : 0;
}

size_t prune_scratch_bytes(int W, int H) {
  const size_t n = (size_t)W * H;
  const size_t blocks = (n + kPruneBlock - 1) / kPruneBlock;
  const size_t counts = (2 * blocks + 1) * sizeof(uint32_t);
  return ((counts + 255) / 256) * 256 + ((n + 255) / 256) * 256;
}

cudaError_t launch_prune(const PruneView* d_views, int n_views, int W, int H, float thr,
                         void* scratch, PruneOut out, unsigned long long* d_count,
                         cudaStream_t s) {
  const size_t n = (size_t)W * H;
  const int blocks = (int)((n + kPruneBlock - 1) / kPruneBlock);
  uint32_t* counts = static_cast<uint32_t*>(scratch);
  uint32_t* offsets = counts + blocks;
  const size_t counts_bytes = ((((2 * (size_t)blocks + 1) * sizeof(uint32_t)) + 255) / 256) * 256;
  uint8_t* keep = static_cast<uint8_t*>(scratch) + counts_bytes;
  prune_flags_kernel<<<blocks, kPruneBlock, 0, s>>>(d_views, n_views, thr, keep, counts);
  scan_counts_kernel<<<1, 1024, 0, s>>>(counts, blocks, offsets, d_count);
  if (out.points)
    prune_write_kernel<<<blocks, kPruneBlock, 0, s>>>(d_views, n_views, thr, keep, offsets, out);
  return cudaGetLastError();
}

}  // namespace dn
