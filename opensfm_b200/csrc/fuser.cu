// DepthmapFuser (fuser.h:28-77, fuser.cc:35-482): per-pixel fusion of
// depthmaps into a point cloud, then statistical outlier removal.
//
// The reference fuses primary views one after another; within a view it
// walks the pixels in raster order, and every fused pixel marks itself and
// the source pixels it used, which later pixels then skip.  Only that
// marking is sequential.  Everything else a pixel needs -- its world point
// and normal, and for each neighbour the projection, the bilinear source
// depth, the asymmetric depth test, the forward-backward reprojection test
// and the normal test -- depends on the inputs alone.  So the GPU computes,
// for every pixel of a primary view and every neighbour, the candidate
// observation (source pixel, world point, world normal) in one launch; the
// host walks the pixels in the reference's order and applies the marks; and
// the GPU takes the component-wise medians of the surviving observations.
//
// Arithmetic is FP32 in the order of the reference's expressions, every
// operation rounded by itself (no contraction), with the 3x3 inverses in
// Eigen's cofactor order; the result is the single-thread result of the
// reference.  The statistical outlier removal (fuser.cc:374-482) follows
// at the end of the file.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "dense_b200.h"
#include "device_guard.h"

namespace {

thread_local std::string g_fuse_error;

dn_status ffail(dn_status s, const std::string& m) {
  g_fuse_error = m;
  return s;
}

#define FCHECK(cond, msg) \
  do {                    \
    if (!(cond)) return ffail(DN_INVALID_ARG, msg); \
  } while (0)
#define FCUDA(expr)                                                        \
  do {                                                                     \
    cudaError_t e_ = (expr);                                               \
    if (e_ != cudaSuccess) {                                               \
      return ffail(e_ == cudaErrorMemoryAllocation ? DN_OUT_OF_MEMORY      \
                                                   : DN_DEVICE_ERROR,      \
                   cudaGetErrorString(e_));                                \
    }                                                                      \
  } while (0)

struct FCam {
  float K[9], Kinv[9], R[9], t[3];
};

// Eigen's 3x3 inverse: cofactors, determinant from the first column,
// inverse(j, i) = cof(i, j) * (1 / det).
void inv3_eigen(const float* m, float* o) {
  float cof[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
      cof[3 * i + j] = m[3 * i1 + j1] * m[3 * i2 + j2] - m[3 * i1 + j2] * m[3 * i2 + j1];
    }
  const float det = (m[0] * cof[0] + m[3] * cof[3]) + m[6] * cof[6];
  const float invdet = 1.0f / det;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) o[3 * j + i] = cof[3 * i + j] * invdet;
}

struct ViewDevF {
  FCam cam;
  int W, H;
  const float* depth;    // [H][W]
  const float* normal;   // [H][W][3]
  const uint8_t* mask;   // [H][W] or null
  const uint8_t* fused;  // [H][W] marks as of the start of the current view
  const uint8_t* color;  // [H][W][3]
};

// One observation handed to the host: the reference pixel's own (view
// slot -1, pix = its index) followed by its neighbours' (slot k, pix = the
// source pixel), in raster order of the reference pixels.
struct FuseRec {
  int slot, pix;
  float pt[3], nrm[3];
};

struct Params {
  float max_reproj_sq, max_depth_error, min_cos, behind;
  int border;
};

// ---------------------------------------------------------------- device
__device__ inline void mv(const float* m, float x, float y, float z, float* o) {
  o[0] = __fadd_rn(__fadd_rn(__fmul_rn(m[0], x), __fmul_rn(m[1], y)), __fmul_rn(m[2], z));
  o[1] = __fadd_rn(__fadd_rn(__fmul_rn(m[3], x), __fmul_rn(m[4], y)), __fmul_rn(m[5], z));
  o[2] = __fadd_rn(__fadd_rn(__fmul_rn(m[6], x), __fmul_rn(m[7], y)), __fmul_rn(m[8], z));
}
__device__ inline void mtv(const float* m, float x, float y, float z, float* o) {
  o[0] = __fadd_rn(__fadd_rn(__fmul_rn(m[0], x), __fmul_rn(m[3], y)), __fmul_rn(m[6], z));
  o[1] = __fadd_rn(__fadd_rn(__fmul_rn(m[1], x), __fmul_rn(m[4], y)), __fmul_rn(m[7], z));
  o[2] = __fadd_rn(__fadd_rn(__fmul_rn(m[2], x), __fmul_rn(m[5], y)), __fmul_rn(m[8], z));
}
// R^T (d K^-1 (u, v, 1) - t), with (d K^-1) formed first as Eigen does.
__device__ inline void backproject(const FCam& c, float d, float u, float v, float* o) {
  float m[9], q[3];
#pragma unroll
  for (int i = 0; i < 9; ++i) m[i] = __fmul_rn(d, c.Kinv[i]);
  mv(m, u, v, 1.0f, q);
  mtv(c.R, __fsub_rn(q[0], c.t[0]), __fsub_rn(q[1], c.t[1]), __fsub_rn(q[2], c.t[2]), o);
}
// K (R X + t).
__device__ inline void project(const FCam& c, const float* X, float* o) {
  float p[3];
  mv(c.R, X[0], X[1], X[2], p);
  mv(c.K, __fadd_rn(p[0], c.t[0]), __fadd_rn(p[1], c.t[1]), __fadd_rn(p[2], c.t[2]), o);
}
__device__ inline float norm3(const float* n) {
  return __fsqrt_rn(
      __fadd_rn(__fadd_rn(__fmul_rn(n[0], n[0]), __fmul_rn(n[1], n[1])), __fmul_rn(n[2], n[2])));
}
// BilinearDepth (fuser.cc:95-113) over foundation::BilinearInterpolation
// (foundation/interpolation.h:16-33): -1 outside or next to a depth <= 0.
__device__ inline float bilinear_depth(const float* d, int W, int H, float u, float v) {
  const int x0 = (int)floorf(u), y0 = (int)floorf(v), x1 = x0 + 1, y1 = y0 + 1;
  if (x0 < 0 || y0 < 0 || x1 >= W || y1 >= H) return -1.0f;
  if (d[(size_t)y0 * W + x0] <= 0.0f || d[(size_t)y0 * W + x1] <= 0.0f ||
      d[(size_t)y1 * W + x0] <= 0.0f || d[(size_t)y1 * W + x1] <= 0.0f)
    return -1.0f;
  if (u < 0.0f || u >= (float)(W - 1) || v < 0.0f || v >= (float)(H - 1)) return -1.0f;
  const int ix = (int)u, iy = (int)v;
  const float dx = __fsub_rn(u, (float)ix), dy = __fsub_rn(v, (float)iy);
  const float gx = __fsub_rn(1.0f, dx), gy = __fsub_rn(1.0f, dy);
  const float* p = d + (size_t)iy * W + ix;
  const float v0 = __fadd_rn(__fmul_rn(gx, p[0]), __fmul_rn(dx, p[1]));
  const float v1 = __fadd_rn(__fmul_rn(gx, p[W]), __fmul_rn(dx, p[W + 1]));
  return __fadd_rn(__fmul_rn(gy, v0), __fmul_rn(dy, v1));
}

// One thread per pixel of the reference view `ri`.  ref_pt / ref_nrm are
// written for pixels that can be fused (inside the border margin, mask set,
// depth > 0, normal non-zero; ref_ok = 1).  For neighbour k, cand_pix is
// the source pixel (index in its view) of a consistent observation or -1,
// cand_pt / cand_nrm its world point and normal.
__global__ void fuse_candidates_kernel(const ViewDevF* __restrict__ views, int n_views, int ri,
                                       const int* __restrict__ nbrs, int n_nbrs, Params p,
                                       uint8_t* __restrict__ ref_ok, float* __restrict__ ref_pt,
                                       float* __restrict__ ref_nrm, int* __restrict__ cand_pix,
                                       float* __restrict__ cand_pt, float* __restrict__ cand_nrm,
                                       unsigned* __restrict__ n_rec) {
  const ViewDevF& ref = views[ri];
  const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y * blockDim.y + threadIdx.y;
  if (c >= ref.W || r >= ref.H) return;
  const size_t rp = (size_t)r * ref.W + c;
  const int bm = p.border;
  bool ok = r >= bm && r < ref.H - bm && c >= bm && c < ref.W - bm;
  ok = ok && !(ref.mask && ref.mask[rp] == 0);
  ok = ok && ref.fused[rp] == 0;  // fused by an earlier view: the host skips it
  const float rd = ref.depth[rp];
  ok = ok && rd > 0.0f;
  float rpt[3] = {0.f, 0.f, 0.f}, rnw[3] = {0.f, 0.f, 0.f};
  if (ok) {
    backproject(ref.cam, rd, (float)c, (float)r, rpt);
    const float* rn = ref.normal + 3 * rp;
    const float nl = norm3(rn);
    ok = nl >= 1e-6f;
    if (ok) mtv(ref.cam.R, __fdiv_rn(rn[0], nl), __fdiv_rn(rn[1], nl), __fdiv_rn(rn[2], nl), rnw);
  }
  ref_ok[rp] = ok ? 1 : 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    ref_pt[3 * rp + d] = rpt[d];
    ref_nrm[3 * rp + d] = rnw[d];
  }
  unsigned recs = ok ? 1u : 0u;
  for (int k = 0; k < n_nbrs; ++k) {
    const size_t slot = rp * n_nbrs + k;
    int pix = -1;
    float spt[3] = {0.f, 0.f, 0.f}, snw[3] = {0.f, 0.f, 0.f};
    const int si = nbrs[k];
    if (ok && si >= 0 && si < n_views) {
      const ViewDevF& src = views[si];
      float proj[3];
      project(src.cam, rpt, proj);
      if (proj[2] >= 1e-6f) {
        const float su = __fdiv_rn(proj[0], proj[2]), sv = __fdiv_rn(proj[1], proj[2]);
        if (fabsf(su) < 1e9f && fabsf(sv) < 1e9f) {
          const int scol = (int)roundf(su), srow = (int)roundf(sv);
          if (scol >= bm && scol < src.W - bm && srow >= bm && srow < src.H - bm) {
            const size_t sp = (size_t)srow * src.W + scol;
            // A source pixel marked before this view stays marked: drop it.
            if (!(src.mask && src.mask[sp] == 0) && src.fused[sp] == 0) {
              float sd = bilinear_depth(src.depth, src.W, src.H, su, sv);
              if (sd <= 0.0f) sd = src.depth[sp];
              if (sd > 0.0f) {
                const float front = __fmul_rn(p.max_depth_error, proj[2]);
                const float back = __fmul_rn(front, p.behind);
                const float diff = __fsub_rn(sd, proj[2]);
                if (!(diff > front || diff < -back)) {
                  float rep[3];
                  backproject(src.cam, sd, (float)scol, (float)srow, spt);
                  project(ref.cam, spt, rep);
                  if (rep[2] >= 1e-6f) {
                    const float ex = __fsub_rn(__fdiv_rn(rep[0], rep[2]), (float)c);
                    const float ey = __fsub_rn(__fdiv_rn(rep[1], rep[2]), (float)r);
                    if (!(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)) > p.max_reproj_sq)) {
                      const float* sn = src.normal + 3 * sp;
                      const float sl = norm3(sn);
                      if (sl >= 1e-6f) {
                        mtv(src.cam.R, __fdiv_rn(sn[0], sl), __fdiv_rn(sn[1], sl),
                            __fdiv_rn(sn[2], sl), snw);
                        const float cs = __fadd_rn(
                            __fadd_rn(__fmul_rn(rnw[0], snw[0]), __fmul_rn(rnw[1], snw[1])),
                            __fmul_rn(rnw[2], snw[2]));
                        if (!(cs < p.min_cos)) pix = (int)sp;
                      }
                    }
                  }
                }
              }
            }
          }
        }
      }
    }
    cand_pix[slot] = pix;
    recs += pix >= 0 ? 1u : 0u;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      cand_pt[3 * slot + d] = spt[d];
      cand_nrm[3 * slot + d] = snw[d];
    }
  }
  n_rec[rp] = recs;
}

// Packs each fusable pixel's own observation and its neighbours' into the
// record stream at the pixel's exclusive-scan offset.
__global__ void fuse_compact_kernel(int W, int H, int n_nbrs, const uint8_t* __restrict__ ref_ok,
                                    const float* __restrict__ ref_pt,
                                    const float* __restrict__ ref_nrm,
                                    const int* __restrict__ cand_pix,
                                    const float* __restrict__ cand_pt,
                                    const float* __restrict__ cand_nrm,
                                    const unsigned* __restrict__ offset,
                                    FuseRec* __restrict__ out) {
  const size_t rp = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (rp >= (size_t)W * H || !ref_ok[rp]) return;
  FuseRec* o = out + offset[rp];
  FuseRec r;
  r.slot = -1;
  r.pix = (int)rp;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    r.pt[d] = ref_pt[3 * rp + d];
    r.nrm[d] = ref_nrm[3 * rp + d];
  }
  *o++ = r;
  for (int k = 0; k < n_nbrs; ++k) {
    const size_t slot = rp * n_nbrs + k;
    if (cand_pix[slot] < 0) continue;
    r.slot = k;
    r.pix = cand_pix[slot];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      r.pt[d] = cand_pt[3 * slot + d];
      r.nrm[d] = cand_nrm[3 * slot + d];
    }
    *o++ = r;
  }
}

// VectorMedian (fuser.cc:23-31) is the value nth_element puts at n / 2: the
// n/2-th smallest.  Picked here by rank, the first value in record order
// with fewer than n/2 + 1 values below it and at least n/2 + 1 values at
// or below it (the same value; only -0 and +0 could tell two picks apart).
template <typename T, typename Get>
__device__ inline T rank_median(int n, Get get) {
  const int h = n / 2;
  for (int a = 0; a < n; ++a) {
    const T va = get(a);
    int less = 0, le = 0;
    for (int b = 0; b < n; ++b) {
      const T vb = get(b);
      less += vb < va;
      le += !(va < vb);
    }
    if (less <= h && h < le) return va;
  }
  return get(h);  // only with NaN among the values
}

// One thread per fused point: the component-wise medians of its surviving
// observations (fuser.cc:312-346), the normal renormalised when its length
// exceeds 1e-6.  idx[start[i] .. start[i + 1]) lists the point's records,
// its own first.
__global__ void fuse_median_kernel(const FuseRec* __restrict__ rec,
                                   const unsigned* __restrict__ start,
                                   const unsigned* __restrict__ idx, int n_pts,
                                   const ViewDevF* __restrict__ views, int ri,
                                   const int* __restrict__ nbrs, float* __restrict__ out_pt,
                                   float* __restrict__ out_nrm, uint8_t* __restrict__ out_clr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_pts) return;
  const unsigned* ix = idx + start[i];
  const int n = (int)(start[i + 1] - start[i]);
#pragma unroll 1
  for (int d = 0; d < 3; ++d)
    out_pt[3 * i + d] = rank_median<float>(n, [&](int a) { return rec[ix[a]].pt[d]; });
  float mn[3];
#pragma unroll 1
  for (int d = 0; d < 3; ++d)
    mn[d] = rank_median<float>(n, [&](int a) { return rec[ix[a]].nrm[d]; });
  const float ml = __fsqrt_rn(
      __fadd_rn(__fadd_rn(__fmul_rn(mn[0], mn[0]), __fmul_rn(mn[1], mn[1])), __fmul_rn(mn[2], mn[2])));
  if (ml > 1e-6f)
    for (int d = 0; d < 3; ++d) mn[d] = __fdiv_rn(mn[d], ml);
  for (int d = 0; d < 3; ++d) out_nrm[3 * i + d] = mn[d];
  auto color_of = [&](int a, int d) -> uint8_t {
    const FuseRec& r = rec[ix[a]];
    const int v = r.slot < 0 ? ri : nbrs[r.slot];
    return views[v].color[3 * (size_t)r.pix + d];
  };
#pragma unroll 1
  for (int d = 0; d < 3; ++d)
    out_clr[3 * i + d] = rank_median<uint8_t>(n, [&](int a) { return color_of(a, d); });
}

// ------------------------------------------------------- outlier removal
// Statistical outlier removal (fuser.cc:374-482).  The reference takes the
// K + 1 nearest neighbours of each point from a vlfeat kd-forest of one tree
// with no comparison limit (an exact search), skips the point itself and
// averages the float square roots of the K remaining float L2 distances
// (squared distance summed over x, y, z) in ascending order.  That is the
// mean of the K smallest distances to other points, whatever the tie order,
// and it is computed here exactly on a uniform grid: points are sorted by
// cell, each query scans shells of cells around its own until the K-th
// distance is provably below every unscanned cell's distance (with a slack
// for the cell rounding), and the few queries still open after kSorRings
// shells are finished by one warp each over all points.  The statistics,
// the threshold and the filter follow on the host in point order, in double
// as the reference accumulates them.
constexpr int kSorMaxK = 64;
constexpr int kSorRings = 3;

struct SorGrid {
  float ox, oy, oz, h, slack;
  int nx, ny, nz;
};

__device__ inline float sor_d2(float4 q, float4 p) {
  const float dx = __fsub_rn(q.x, p.x), dy = __fsub_rn(q.y, p.y), dz = __fsub_rn(q.z, p.z);
  return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// Keeps best[0 .. cnt) as the smallest values seen, ascending, cnt <= K.
__device__ inline void sor_insert(float* best, int& cnt, int K, float d2) {
  if (cnt == K && !(d2 < best[K - 1])) return;
  int m = cnt < K ? cnt++ : K - 1;
  while (m > 0 && best[m - 1] > d2) {
    best[m] = best[m - 1];
    --m;
  }
  best[m] = d2;
}

__device__ inline int sor_cell(float v, float o, float h, int n) {
  const int c = (int)floorf(__fdiv_rn(__fsub_rn(v, o), h));
  return min(max(c, 0), n - 1);
}

__global__ void sor_keys_kernel(const float* __restrict__ pts, int n, SorGrid g,
                                unsigned long long* __restrict__ key, int* __restrict__ idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int cx = sor_cell(pts[3 * i], g.ox, g.h, g.nx);
  const int cy = sor_cell(pts[3 * i + 1], g.oy, g.h, g.ny);
  const int cz = sor_cell(pts[3 * i + 2], g.oz, g.h, g.nz);
  key[i] = ((unsigned long long)cz * g.ny + cy) * g.nx + cx;
  idx[i] = i;
}

// Points in cell order, the original index in w.
__global__ void sor_gather_kernel(const float* __restrict__ pts, const int* __restrict__ idx,
                                  int n, float4* __restrict__ sp) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const int i = idx[s];
  sp[s] = make_float4(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], __int_as_float(i));
}

__device__ inline int sor_lower_bound(const unsigned long long* __restrict__ a, int n,
                                      unsigned long long v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__device__ inline float sor_mean(const float* best, int K) {
  float sum = 0.0f;
  for (int m = 0; m < K; ++m) sum = __fadd_rn(sum, __fsqrt_rn(best[m]));
  return __fdiv_rn(sum, (float)K);
}

// One thread per point, in cell order.  Writes mean_knn[original index], or
// queues the point for the brute-force pass.
__global__ void sor_knn_kernel(const float4* __restrict__ sp,
                               const unsigned long long* __restrict__ skey, int n, SorGrid g,
                               int K, float* __restrict__ mean_knn, int* __restrict__ open_q,
                               unsigned* __restrict__ n_open) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float4 q = sp[s];
  const int self = __float_as_int(q.w);
  const unsigned long long ck = skey[s];
  const int cx = (int)(ck % (unsigned long long)g.nx);
  const int cy = (int)((ck / (unsigned long long)g.nx) % (unsigned long long)g.ny);
  const int cz = (int)(ck / ((unsigned long long)g.nx * g.ny));
  float best[kSorMaxK];
  int cnt = 0;
  auto scan = [&](int lo, int hi) {
    for (int j = lo; j < hi; ++j) {
      const float4 p = sp[j];
      if (__float_as_int(p.w) == self) continue;
      sor_insert(best, cnt, K, sor_d2(q, p));
    }
  };
  auto key = [&](int x, int y, int z) {
    return ((unsigned long long)z * g.ny + y) * g.nx + x;
  };
  bool done = false;
  for (int r = 0; r <= kSorRings && !done; ++r) {
    for (int dz = -r; dz <= r; ++dz) {
      const int z = cz + dz;
      if (z < 0 || z >= g.nz) continue;
      for (int dy = -r; dy <= r; ++dy) {
        const int y = cy + dy;
        if (y < 0 || y >= g.ny) continue;
        if (abs(dz) == r || abs(dy) == r) {  // a face row: the whole run of x
          const int x0 = max(cx - r, 0), x1 = min(cx + r, g.nx - 1);
          scan(sor_lower_bound(skey, n, key(x0, y, z)), sor_lower_bound(skey, n, key(x1, y, z) + 1));
        } else {  // inside the shell's cross-section: only its two end cells
          for (int e = 0; e < 2; ++e) {
            const int x = e ? cx + r : cx - r;
            if (x >= 0 && x < g.nx)
              scan(sor_lower_bound(skey, n, key(x, y, z)), sor_lower_bound(skey, n, key(x, y, z) + 1));
          }
        }
      }
    }
    // Distance from q to the nearest face of the scanned box that has cells
    // beyond it; none left means every point has been scanned.
    float dmin = INFINITY;
    if (cx - r > 0) dmin = fminf(dmin, q.x - (g.ox + (float)(cx - r) * g.h));
    if (cx + r < g.nx - 1) dmin = fminf(dmin, (g.ox + (float)(cx + r + 1) * g.h) - q.x);
    if (cy - r > 0) dmin = fminf(dmin, q.y - (g.oy + (float)(cy - r) * g.h));
    if (cy + r < g.ny - 1) dmin = fminf(dmin, (g.oy + (float)(cy + r + 1) * g.h) - q.y);
    if (cz - r > 0) dmin = fminf(dmin, q.z - (g.oz + (float)(cz - r) * g.h));
    if (cz + r < g.nz - 1) dmin = fminf(dmin, (g.oz + (float)(cz + r + 1) * g.h) - q.z);
    if (dmin == INFINITY) {
      done = true;
    } else {
      dmin -= g.slack;
      done = cnt == K && dmin > 0.0f && best[K - 1] <= dmin * dmin * (1.0f - 1e-5f);
    }
  }
  if (done && cnt == K)
    mean_knn[self] = sor_mean(best, K);
  else
    open_q[atomicAdd(n_open, 1u)] = s;
}

// One warp per open query: every lane keeps the K smallest distances of its
// stride over all points; K rounds of a warp-wide minimum then merge them in
// ascending order.
__global__ void sor_brute_kernel(const float4* __restrict__ sp, int n,
                                 const int* __restrict__ open_q, int n_open, int K,
                                 float* __restrict__ mean_knn) {
  const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= n_open) return;  // whole warps leave together
  const float4 q = sp[open_q[w]];
  const int self = __float_as_int(q.w);
  float best[kSorMaxK];
  int cnt = 0;
  for (int j = lane; j < n; j += 32) {
    const float4 p = sp[j];
    if (__float_as_int(p.w) == self) continue;
    sor_insert(best, cnt, K, sor_d2(q, p));
  }
  int head = 0;
  float sum = 0.0f;
  for (int m = 0; m < K; ++m) {
    const float v = head < cnt ? best[head] : INFINITY;
    float mv = v;
    int ml = lane;
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, mv, o);
      const int ol = __shfl_xor_sync(0xffffffffu, ml, o);
      if (ov < mv || (ov == mv && ol < ml)) {
        mv = ov;
        ml = ol;
      }
    }
    if (lane == ml) ++head;
    sum = __fadd_rn(sum, __fsqrt_rn(mv));
  }
  if (lane == 0) mean_knn[self] = __fdiv_rn(sum, (float)K);
}

// ------------------------------------------------------------------ host
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    if (count <= n && p) return cudaSuccess;
    release();
    if (!count) return cudaSuccess;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e == cudaSuccess) n = count;
    return e;
  }
};
template <typename T>
struct HBuf {  // pinned host buffer
  T* p = nullptr;
  size_t n = 0;
  HBuf() = default;
  HBuf(const HBuf&) = delete;
  HBuf& operator=(const HBuf&) = delete;
  ~HBuf() {
    if (p) cudaFreeHost(p);
  }
  cudaError_t alloc(size_t count) {
    if (count <= n && p) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e == cudaSuccess) n = count;
    return e;
  }
};

struct FView {
  FCam cam;
  int W = 0, H = 0;
  std::vector<int> nbrs;
  bool primary = true;
  bool has_mask = false;
  DBuf<float> depth, normal;
  DBuf<uint8_t> mask, color;
};

}  // namespace

struct dn_fuser {
  int device = 0;
  cudaStream_t stream = nullptr;
  int min_num_consistent = 3;
  float max_reproj_error_sq = 4.0f;
  float max_depth_error = 0.01f;
  float max_normal_deg = 10.0f;
  int border = 5;
  float behind = 0.3f;
  int sor_knn = 12;  // the reference's defaults (fuser.cc:45-46)
  float sor_factor = 2.5f;
  float sor_ms = 0.0f;  // device time of the last outlier removal
  std::vector<std::unique_ptr<FView>> views;
  std::vector<float> out_pts, out_nrm;
  std::vector<uint8_t> out_clr;
  ~dn_fuser() {
    if (stream) cudaStreamDestroy(stream);
  }
};

extern "C" const char* dn_fuser_last_error(void) { return g_fuse_error.c_str(); }

extern "C" dn_status dn_fuser_create(dn_fuser** out) {
  const dn::DeviceRestore device_restore_;
  FCHECK(out, "NULL output");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return ffail(DN_DEVICE_ERROR, "no CUDA device");
  auto f = std::make_unique<dn_fuser>();
  FCUDA(cudaGetDevice(&f->device));
  FCUDA(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking));
  *out = f.release();
  return DN_OK;
}
extern "C" dn_status dn_fuser_destroy(dn_fuser* f) {
  const dn::DeviceRestore device_restore_;
  delete f;
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_min_num_consistent(dn_fuser* f, int n) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f, "NULL fuser");
  f->min_num_consistent = n;
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_max_reproj_error(dn_fuser* f, float px) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f, "NULL fuser");
  f->max_reproj_error_sq = px * px;  // fuser.cc:57-59
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_max_depth_error(dn_fuser* f, float ratio) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f, "NULL fuser");
  f->max_depth_error = ratio;
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_max_normal_error(dn_fuser* f, float degrees) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f, "NULL fuser");
  f->max_normal_deg = degrees;
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_border_margin(dn_fuser* f, int px) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f, "NULL fuser");
  f->border = std::max(0, px);  // fuser.cc:67-69
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_sor_params(dn_fuser* f, int knn, float stddev_factor) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f, "NULL fuser");
  FCHECK(knn <= kSorMaxK, "knn above 64 is not supported");
  f->sor_knn = std::max(0, knn);  // knn <= 0 skips the step, as the reference does
  f->sor_factor = stddev_factor;
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_behind_depth_factor(dn_fuser* f, float factor) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f, "NULL fuser");
  f->behind = std::min(1.0f, std::max(0.0f, factor));  // fuser.cc:78-80
  return DN_OK;
}

extern "C" dn_status dn_fuser_add_view(dn_fuser* f, const double* K, const double* R,
                                       const double* t, const float* depth, const float* normal,
                                       const uint8_t* color, const uint8_t* mask, int width,
                                       int height, const int* neighbor_ids, int n_neighbors,
                                       int primary) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f, "NULL fuser");
  FCHECK(K && R && t && depth && normal && color, "NULL argument");
  FCHECK(width >= 1 && height >= 1 && width <= 16384 && height <= 16384, "bad depthmap size");
  FCHECK(n_neighbors >= 0 && n_neighbors <= 1024 && (n_neighbors == 0 || neighbor_ids),
         "neighbour list must hold 0..1024 ids");
  for (int i = 0; i < 9; ++i) FCHECK(std::isfinite(K[i]) && std::isfinite(R[i]), "K, R must be finite");
  for (int i = 0; i < 3; ++i) FCHECK(std::isfinite(t[i]), "t must be finite");
  FCUDA(cudaSetDevice(f->device));
  auto v = std::make_unique<FView>();
  for (int i = 0; i < 9; ++i) {
    v->cam.K[i] = (float)K[i];
    v->cam.R[i] = (float)R[i];
  }
  for (int i = 0; i < 3; ++i) v->cam.t[i] = (float)t[i];
  inv3_eigen(v->cam.K, v->cam.Kinv);
  v->W = width;
  v->H = height;
  const size_t npx = (size_t)width * height;
  v->nbrs.assign(neighbor_ids, neighbor_ids + n_neighbors);
  v->primary = primary != 0;
  FCUDA(v->depth.alloc(npx));
  FCUDA(v->normal.alloc(3 * npx));
  FCUDA(v->color.alloc(3 * npx));
  FCUDA(cudaMemcpyAsync(v->color.p, color, 3 * npx, cudaMemcpyHostToDevice, f->stream));
  FCUDA(cudaMemcpyAsync(v->depth.p, depth, npx * sizeof(float), cudaMemcpyHostToDevice, f->stream));
  FCUDA(cudaMemcpyAsync(v->normal.p, normal, 3 * npx * sizeof(float), cudaMemcpyHostToDevice,
                        f->stream));
  if (mask) {
    v->has_mask = true;
    FCUDA(v->mask.alloc(npx));
    FCUDA(cudaMemcpyAsync(v->mask.p, mask, npx, cudaMemcpyHostToDevice, f->stream));
  }
  FCUDA(cudaStreamSynchronize(f->stream));
  f->views.push_back(std::move(v));
  return DN_OK;
}

// Mean distance to the K nearest other points (fuser.cc:405-438) for each
// of the N points P (xyz rows), on the device; mk receives them in point
// order, *ms the device time.  Requires N > K + 1 and 1 <= K <= kSorMaxK.
static dn_status sor_mean_knn(cudaStream_t s, const float* P, size_t N, int K,
                              std::vector<float>& mk, float* ms) {
  FCHECK(N < (size_t(1) << 31), "too many points for the outlier removal");
  const int n = (int)N;
  // Grid over the bounding box: cell edge from the volume per point, K + 1
  // points to a cell on average if they filled the box, halved because
  // surface points are denser than that where they lie.
  float lo[3] = {P[0], P[1], P[2]}, hi[3] = {P[0], P[1], P[2]};
  float amax = 0.0f;
  for (size_t i = 0; i < N; ++i)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], P[3 * i + d]);
      hi[d] = std::max(hi[d], P[3 * i + d]);
      amax = std::max(amax, std::fabs(P[3 * i + d]));
    }
  FCHECK(std::isfinite(amax), "points must be finite for the outlier removal");
  double ext[3], emax = 0.0;
  for (int d = 0; d < 3; ++d) {
    ext[d] = (double)hi[d] - (double)lo[d];
    emax = std::max(emax, ext[d]);
  }
  const double floor_ext = std::max(emax * 1e-3, 1e-6);
  const double vol = std::max(ext[0], floor_ext) * std::max(ext[1], floor_ext) *
                     std::max(ext[2], floor_ext);
  double h = 0.5 * std::cbrt(vol * (K + 1) / (double)N);
  h = std::max(h, std::max(emax, 1e-6) / (double)(1 << 20));  // at most 2^20 cells an axis
  SorGrid g;
  g.ox = lo[0];
  g.oy = lo[1];
  g.oz = lo[2];
  g.h = (float)h;
  g.nx = (int)(ext[0] / h) + 1;
  g.ny = (int)(ext[1] / h) + 1;
  g.nz = (int)(ext[2] / h) + 1;
  // Cell rounding moves a point across a face by a few ULPs of its
  // coordinates at most; the bound keeps a far wider margin.
  g.slack = (float)(1e-5 * ((double)amax + h));

  cudaEvent_t e0, e1;
  FCUDA(cudaEventCreate(&e0));
  FCUDA(cudaEventCreate(&e1));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } evg{e0, e1};
  DBuf<float> d_pts, d_mean;
  DBuf<unsigned long long> d_key, d_skey;
  DBuf<int> d_idx, d_sidx, d_open;
  DBuf<float4> d_sp;
  DBuf<unsigned> d_nopen;
  DBuf<uint8_t> d_tmp;
  FCUDA(d_pts.alloc(3 * N));
  FCUDA(d_mean.alloc(N));
  FCUDA(d_key.alloc(N));
  FCUDA(d_skey.alloc(N));
  FCUDA(d_idx.alloc(N));
  FCUDA(d_sidx.alloc(N));
  FCUDA(d_open.alloc(N));
  FCUDA(d_sp.alloc(N));
  FCUDA(d_nopen.alloc(1));
  FCUDA(cudaMemcpyAsync(d_pts.p, P, 3 * N * sizeof(float), cudaMemcpyHostToDevice, s));
  FCUDA(cudaEventRecord(e0, s));
  FCUDA(cudaMemsetAsync(d_nopen.p, 0, sizeof(unsigned), s));
  const unsigned blocks = (unsigned)((N + 255) / 256);
  sor_keys_kernel<<<blocks, 256, 0, s>>>(d_pts.p, n, g, d_key.p, d_idx.p);
  FCUDA(cudaGetLastError());
  size_t tmp_bytes = 0;
  FCUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_key.p, d_skey.p, d_idx.p, d_sidx.p,
                                        n, 0, 64, s));
  FCUDA(d_tmp.alloc(std::max<size_t>(tmp_bytes, 1)));
  FCUDA(cub::DeviceRadixSort::SortPairs(d_tmp.p, tmp_bytes, d_key.p, d_skey.p, d_idx.p,
                                        d_sidx.p, n, 0, 64, s));
  sor_gather_kernel<<<blocks, 256, 0, s>>>(d_pts.p, d_sidx.p, n, d_sp.p);
  FCUDA(cudaGetLastError());
  sor_knn_kernel<<<(unsigned)((N + 127) / 128), 128, 0, s>>>(d_sp.p, d_skey.p, n, g, K,
                                                             d_mean.p, d_open.p, d_nopen.p);
  FCUDA(cudaGetLastError());
  unsigned n_open = 0;
  FCUDA(cudaMemcpyAsync(&n_open, d_nopen.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  FCUDA(cudaStreamSynchronize(s));
  if (n_open) {
    const unsigned warps_per_block = 4;
    sor_brute_kernel<<<(n_open + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0,
                       s>>>(d_sp.p, n, d_open.p, (int)n_open, K, d_mean.p);
    FCUDA(cudaGetLastError());
  }
  FCUDA(cudaEventRecord(e1, s));
  mk.resize(N);
  FCUDA(cudaMemcpyAsync(mk.data(), d_mean.p, N * sizeof(float), cudaMemcpyDeviceToHost, s));
  FCUDA(cudaStreamSynchronize(s));
  FCUDA(cudaEventElapsedTime(ms, e0, e1));
  return DN_OK;
}

// The reference's statistics over the means (fuser.cc:442-455): double
// sums in point order, threshold mean + factor * std rounded to float.
static float sor_threshold(const std::vector<float>& mk, float factor) {
  double sum_d = 0.0, sum_d2 = 0.0;
  for (size_t i = 0; i < mk.size(); ++i) {
    const double d = mk[i];
    if (d < 1e20f) {
      sum_d += d;
      sum_d2 += d * d;
    }
  }
  const double mean_d = sum_d / (double)mk.size();
  const double var_d = sum_d2 / (double)mk.size() - mean_d * mean_d;
  const double std_d = std::sqrt(std::max(0.0, var_d));
  return (float)(mean_d + factor * std_d);
}

// The outlier removal over the fused points (fuser.cc:374-482).
static dn_status run_sor(dn_fuser* f) {
  const int K = f->sor_knn;
  const size_t N = f->out_pts.size() / 3;
  f->sor_ms = 0.0f;
  if (K <= 0 || N <= (size_t)K + 1) return DN_OK;
  std::vector<float> mk;
  const dn_status st = sor_mean_knn(f->stream, f->out_pts.data(), N, K, mk, &f->sor_ms);
  if (st != DN_OK) return st;
  const float threshold = sor_threshold(mk, f->sor_factor);
  size_t kept = 0;
  for (size_t i = 0; i < N; ++i) {
    if (!(mk[i] <= threshold)) continue;
    if (kept != i) {
      std::memcpy(&f->out_pts[3 * kept], &f->out_pts[3 * i], 3 * sizeof(float));
      std::memcpy(&f->out_nrm[3 * kept], &f->out_nrm[3 * i], 3 * sizeof(float));
      std::memcpy(&f->out_clr[3 * kept], &f->out_clr[3 * i], 3);
    }
    ++kept;
  }
  f->out_pts.resize(3 * kept);
  f->out_nrm.resize(3 * kept);
  f->out_clr.resize(3 * kept);
  return DN_OK;
}

extern "C" dn_status dn_sor_filter(const float* points, int64_t n, int knn, float stddev_factor,
                                   uint8_t* keep, float* mean_knn) {
  const dn::DeviceRestore device_restore_;
  FCHECK(n >= 0 && (n == 0 || points) && (n == 0 || keep), "NULL argument");
  FCHECK(knn <= kSorMaxK, "knn above 64 is not supported");
  if (knn <= 0 || n <= (int64_t)knn + 1) {
    std::memset(keep, 1, (size_t)n);
    return DN_OK;
  }
  int dev = 0;
  FCUDA(cudaGetDevice(&dev));
  cudaStream_t s;
  FCUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{s};
  std::vector<float> mk;
  float ms = 0.0f;
  const dn_status st = sor_mean_knn(s, points, (size_t)n, knn, mk, &ms);
  if (st != DN_OK) return st;
  const float threshold = sor_threshold(mk, stddev_factor);
  for (int64_t i = 0; i < n; ++i) keep[i] = mk[i] <= threshold ? 1 : 0;
  if (mean_knn) std::memcpy(mean_knn, mk.data(), (size_t)n * sizeof(float));
  return DN_OK;
}

extern "C" dn_status dn_fuser_last_removal_ms(dn_fuser* f, float* ms) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f && ms, "NULL argument");
  *ms = f->sor_ms;
  return DN_OK;
}

extern "C" dn_status dn_fuser_fuse(dn_fuser* f, int64_t* count) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f && count, "NULL argument");
  *count = 0;
  f->out_pts.clear();
  f->out_nrm.clear();
  f->out_clr.clear();
  const int nv = (int)f->views.size();
  if (nv == 0) return DN_OK;
  FCUDA(cudaSetDevice(f->device));
  std::vector<ViewDevF> hv(nv);
  for (int i = 0; i < nv; ++i) {
    const FView& v = *f->views[i];
    hv[i].cam = v.cam;
    hv[i].W = v.W;
    hv[i].H = v.H;
    hv[i].depth = v.depth.p;
    hv[i].normal = v.normal.p;
    hv[i].mask = v.has_mask ? v.mask.p : nullptr;
    hv[i].color = v.color.p;
  }
  DBuf<ViewDevF> d_views;
  FCUDA(d_views.alloc(nv));
  Params p;
  p.max_reproj_sq = f->max_reproj_error_sq;
  p.max_depth_error = f->max_depth_error;
  p.min_cos = std::cos(f->max_normal_deg * static_cast<float>(M_PI) / 180.0f);
  p.behind = f->behind;
  p.border = f->border;

  // Fused marks: host copy (pinned, written by the raster walk) and device
  // copy (read by the candidate kernel), one byte per pixel of every view.
  std::vector<size_t> moff(nv + 1, 0);
  for (int i = 0; i < nv; ++i) moff[i + 1] = moff[i] + (size_t)f->views[i]->W * f->views[i]->H;
  HBuf<uint8_t> h_marks;
  DBuf<uint8_t> d_marks;
  FCUDA(h_marks.alloc(moff[nv]));
  FCUDA(d_marks.alloc(moff[nv]));
  std::memset(h_marks.p, 0, moff[nv]);
  FCUDA(cudaMemsetAsync(d_marks.p, 0, moff[nv], f->stream));
  std::vector<uint8_t> dirty(nv, 0);
  for (int i = 0; i < nv; ++i) hv[i].fused = d_marks.p + moff[i];
  FCUDA(cudaMemcpyAsync(d_views.p, hv.data(), nv * sizeof(ViewDevF), cudaMemcpyHostToDevice,
                        f->stream));

  DBuf<int> d_nbrs;
  DBuf<uint8_t> d_ok;
  DBuf<float> d_rpt, d_rnrm, d_cpt, d_cnrm;
  DBuf<int> d_cpix;
  DBuf<unsigned> d_nrec, d_off;
  DBuf<FuseRec> d_rec;
  DBuf<uint8_t> d_scan_tmp;
  HBuf<FuseRec> h_rec;
  HBuf<unsigned> h_tail;
  FCUDA(h_tail.alloc(2));
  // Sized once: the median kernel of one view may still read it when the
  // next view's list is queued behind it.
  size_t max_nn = 1;
  for (int i = 0; i < nv; ++i) {
    const FView& v = *f->views[i];
    max_nn = std::max(max_nn, v.nbrs.size());
    // Record counts and offsets are 32-bit.
    FCHECK(!v.primary || (size_t)v.W * v.H * (1 + v.nbrs.size()) < (size_t(1) << 32),
           "primary view too large for its neighbour count");
  }
  FCUDA(d_nbrs.alloc(max_nn));
  // Per fused point of the current view: its records (start / idx), and the
  // medians the GPU computes from them, staged for the host.
  HBuf<unsigned> h_start, h_idx;
  DBuf<unsigned> d_start, d_idx;
  DBuf<float> d_vpt, d_vnrm;
  DBuf<uint8_t> d_vclr;
  HBuf<float> h_vpt, h_vnrm;
  HBuf<uint8_t> h_vclr;
  size_t staged = 0;  // points of the previous view in h_v*, not yet appended
  auto append_staged = [&]() {
    f->out_pts.insert(f->out_pts.end(), h_vpt.p, h_vpt.p + 3 * staged);
    f->out_nrm.insert(f->out_nrm.end(), h_vnrm.p, h_vnrm.p + 3 * staged);
    f->out_clr.insert(f->out_clr.end(), h_vclr.p, h_vclr.p + 3 * staged);
    staged = 0;
  };

  for (int ri = 0; ri < nv; ++ri) {
    const FView& ref = *f->views[ri];
    if (!ref.primary) continue;
    const int nn = (int)ref.nbrs.size();
    const size_t npx = (size_t)ref.W * ref.H;
    const size_t nslot = npx * (size_t)std::max(nn, 1);
    // Marks set by earlier views, for the views this one reads.
    auto push_marks = [&](int v) -> cudaError_t {
      if (v < 0 || v >= nv || !dirty[v]) return cudaSuccess;
      dirty[v] = 0;
      return cudaMemcpyAsync(d_marks.p + moff[v], h_marks.p + moff[v], moff[v + 1] - moff[v],
                             cudaMemcpyHostToDevice, f->stream);
    };
    FCUDA(push_marks(ri));
    for (int k = 0; k < nn; ++k) FCUDA(push_marks(ref.nbrs[k]));
    if (nn)
      FCUDA(cudaMemcpyAsync(d_nbrs.p, ref.nbrs.data(), nn * sizeof(int), cudaMemcpyHostToDevice,
                            f->stream));
    FCUDA(d_ok.alloc(npx));
    FCUDA(d_rpt.alloc(3 * npx));
    FCUDA(d_rnrm.alloc(3 * npx));
    FCUDA(d_cpix.alloc(nslot));
    FCUDA(d_cpt.alloc(3 * nslot));
    FCUDA(d_cnrm.alloc(3 * nslot));
    FCUDA(d_nrec.alloc(npx));
    FCUDA(d_off.alloc(npx));
    const dim3 blk(32, 8), grid((ref.W + 31) / 32, (ref.H + 7) / 8);
    fuse_candidates_kernel<<<grid, blk, 0, f->stream>>>(d_views.p, nv, ri, d_nbrs.p, nn, p,
                                                        d_ok.p, d_rpt.p, d_rnrm.p, d_cpix.p,
                                                        d_cpt.p, d_cnrm.p, d_nrec.p);
    FCUDA(cudaGetLastError());
    // Record offsets: exclusive scan of the per-pixel record counts.
    size_t tmp_bytes = 0;
    FCUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_nrec.p, d_off.p, (int)npx,
                                        f->stream));
    FCUDA(d_scan_tmp.alloc(std::max<size_t>(tmp_bytes, 1)));
    FCUDA(cub::DeviceScan::ExclusiveSum(d_scan_tmp.p, tmp_bytes, d_nrec.p, d_off.p, (int)npx,
                                        f->stream));
    FCUDA(cudaMemcpyAsync(h_tail.p, d_off.p + npx - 1, sizeof(unsigned), cudaMemcpyDeviceToHost,
                          f->stream));
    FCUDA(cudaMemcpyAsync(h_tail.p + 1, d_nrec.p + npx - 1, sizeof(unsigned),
                          cudaMemcpyDeviceToHost, f->stream));
    FCUDA(cudaStreamSynchronize(f->stream));
    append_staged();  // the previous view's medians arrived before the tail
    const size_t n_rec = (size_t)h_tail.p[0] + h_tail.p[1];
    if (!n_rec) continue;
    FCUDA(d_rec.alloc(n_rec));
    FCUDA(h_rec.alloc(n_rec));
    FCUDA(h_idx.alloc(n_rec));
    FCUDA(h_start.alloc(n_rec + 1));
    fuse_compact_kernel<<<(unsigned)((npx + 255) / 256), 256, 0, f->stream>>>(
        ref.W, ref.H, nn, d_ok.p, d_rpt.p, d_rnrm.p, d_cpix.p, d_cpt.p, d_cnrm.p, d_off.p,
        d_rec.p);
    FCUDA(cudaGetLastError());
    FCUDA(cudaMemcpyAsync(h_rec.p, d_rec.p, n_rec * sizeof(FuseRec), cudaMemcpyDeviceToHost,
                          f->stream));
    FCUDA(cudaStreamSynchronize(f->stream));

    // The reference's raster walk over the records (fuser.cc:163-355): a
    // pixel's own record (slot -1) opens its run; a pixel or source pixel
    // marked earlier is skipped; a pixel with enough observations is fused
    // and marks itself and the source pixels it used.
    uint8_t* rf = h_marks.p + moff[ri];
    size_t q = 0, n_idx = 0;
    size_t n_pts = 0;
    while (q < n_rec) {
      const size_t own = q++;
      const size_t rp = (size_t)h_rec.p[own].pix;
      size_t q_end = q;
      while (q_end < n_rec && h_rec.p[q_end].slot >= 0) ++q_end;
      if (rf[rp]) {
        q = q_end;
        continue;
      }
      const size_t first = n_idx;
      h_idx.p[n_idx++] = (unsigned)own;
      for (; q < q_end; ++q) {
        const FuseRec& o = h_rec.p[q];
        if (h_marks.p[moff[ref.nbrs[o.slot]] + o.pix]) continue;
        h_idx.p[n_idx++] = (unsigned)q;
      }
      if ((int)(n_idx - first) < f->min_num_consistent) {
        n_idx = first;
        continue;
      }
      h_start.p[n_pts++] = (unsigned)first;
      rf[rp] = 1;
      dirty[ri] = 1;
      for (size_t k = first + 1; k < n_idx; ++k) {
        const FuseRec& o = h_rec.p[h_idx.p[k]];
        const int si = ref.nbrs[o.slot];
        h_marks.p[moff[si] + o.pix] = 1;
        dirty[si] = 1;
      }
    }
    if (!n_pts) continue;
    h_start.p[n_pts] = (unsigned)n_idx;
    FCUDA(d_start.alloc(n_pts + 1));
    FCUDA(d_idx.alloc(n_idx));
    FCUDA(d_vpt.alloc(3 * n_pts));
    FCUDA(d_vnrm.alloc(3 * n_pts));
    FCUDA(d_vclr.alloc(3 * n_pts));
    FCUDA(h_vpt.alloc(3 * n_pts));
    FCUDA(h_vnrm.alloc(3 * n_pts));
    FCUDA(h_vclr.alloc(3 * n_pts));
    FCUDA(cudaMemcpyAsync(d_start.p, h_start.p, (n_pts + 1) * sizeof(unsigned),
                          cudaMemcpyHostToDevice, f->stream));
    FCUDA(cudaMemcpyAsync(d_idx.p, h_idx.p, n_idx * sizeof(unsigned), cudaMemcpyHostToDevice,
                          f->stream));
    fuse_median_kernel<<<(unsigned)((n_pts + 127) / 128), 128, 0, f->stream>>>(
        d_rec.p, d_start.p, d_idx.p, (int)n_pts, d_views.p, ri, d_nbrs.p, d_vpt.p, d_vnrm.p,
        d_vclr.p);
    FCUDA(cudaGetLastError());
    FCUDA(cudaMemcpyAsync(h_vpt.p, d_vpt.p, 3 * n_pts * sizeof(float), cudaMemcpyDeviceToHost,
                          f->stream));
    FCUDA(cudaMemcpyAsync(h_vnrm.p, d_vnrm.p, 3 * n_pts * sizeof(float), cudaMemcpyDeviceToHost,
                          f->stream));
    FCUDA(cudaMemcpyAsync(h_vclr.p, d_vclr.p, 3 * n_pts, cudaMemcpyDeviceToHost, f->stream));
    staged = n_pts;
  }
  FCUDA(cudaStreamSynchronize(f->stream));
  append_staged();
  const dn_status st = run_sor(f);
  if (st != DN_OK) return st;
  *count = (int64_t)(f->out_pts.size() / 3);
  return DN_OK;
}

extern "C" dn_status dn_fuser_get(dn_fuser* f, float* points, float* normals, uint8_t* colors,
                                  int64_t capacity) {
  const dn::DeviceRestore device_restore_;
  FCHECK(f, "NULL fuser");
  const int64_t n = (int64_t)(f->out_pts.size() / 3);
  FCHECK(capacity >= n, "capacity below the fused point count");
  if (points) std::memcpy(points, f->out_pts.data(), f->out_pts.size() * sizeof(float));
  if (normals) std::memcpy(normals, f->out_nrm.data(), f->out_nrm.size() * sizeof(float));
  if (colors) std::memcpy(colors, f->out_clr.data(), f->out_clr.size());
  return DN_OK;
}
