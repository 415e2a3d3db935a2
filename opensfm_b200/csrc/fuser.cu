// DepthmapFuser (fuser.h:28-77, fuser.cc:35-372): per-pixel fusion of
// depthmaps into a point cloud.
//
// The reference fuses primary views one after another; within a view it
// walks the pixels in raster order, and every fused pixel marks itself and
// the source pixels it used, which later pixels then skip.  Only that
// marking is sequential.  Everything else a pixel needs -- its world point
// and normal, and for each neighbour the projection, the bilinear source
// depth, the asymmetric depth test, the forward-backward reprojection test
// and the normal test -- depends on the inputs alone.  So the GPU computes,
// for every pixel of a primary view and every neighbour, the candidate
// observation (source pixel, world point, world normal) in one launch, and
// the host walks the pixels in the reference's order, applies the marks,
// and takes the component-wise medians of the surviving observations.
//
// Arithmetic is FP32 in the order of the reference's expressions, every
// operation rounded by itself (no contraction), with the 3x3 inverses in
// Eigen's cofactor order; the result is the single-thread result of the
// reference.  The statistical outlier removal (fuser.cc:374-482) is not
// built: set_sor_params accepts only knn = 0, its setting in OpenSfM's
// dense pipeline (depthmap_fusion_sor_knn = 0).
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "dense_b200.h"

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
  int sor_knn = 0;
  float sor_factor = 2.5f;
  std::vector<std::unique_ptr<FView>> views;
  std::vector<float> out_pts, out_nrm;
  std::vector<uint8_t> out_clr;
  ~dn_fuser() {
    if (stream) cudaStreamDestroy(stream);
  }
};

extern "C" const char* dn_fuser_last_error(void) { return g_fuse_error.c_str(); }

extern "C" dn_status dn_fuser_create(dn_fuser** out) {
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
  delete f;
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_min_num_consistent(dn_fuser* f, int n) {
  FCHECK(f, "NULL fuser");
  f->min_num_consistent = n;
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_max_reproj_error(dn_fuser* f, float px) {
  FCHECK(f, "NULL fuser");
  f->max_reproj_error_sq = px * px;  // fuser.cc:57-59
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_max_depth_error(dn_fuser* f, float ratio) {
  FCHECK(f, "NULL fuser");
  f->max_depth_error = ratio;
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_max_normal_error(dn_fuser* f, float degrees) {
  FCHECK(f, "NULL fuser");
  f->max_normal_deg = degrees;
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_border_margin(dn_fuser* f, int px) {
  FCHECK(f, "NULL fuser");
  f->border = std::max(0, px);  // fuser.cc:67-69
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_sor_params(dn_fuser* f, int knn, float stddev_factor) {
  FCHECK(f, "NULL fuser");
  FCHECK(knn <= 0,
         "statistical outlier removal is not built: knn must be 0 (OpenSfM's dense pipeline "
         "sets depthmap_fusion_sor_knn = 0)");
  f->sor_knn = 0;
  f->sor_factor = stddev_factor;
  return DN_OK;
}
extern "C" dn_status dn_fuser_set_behind_depth_factor(dn_fuser* f, float factor) {
  FCHECK(f, "NULL fuser");
  f->behind = std::min(1.0f, std::max(0.0f, factor));  // fuser.cc:78-80
  return DN_OK;
}

extern "C" dn_status dn_fuser_add_view(dn_fuser* f, const double* K, const double* R,
                                       const double* t, const float* depth, const float* normal,
                                       const uint8_t* color, const uint8_t* mask, int width,
                                       int height, const int* neighbor_ids, int n_neighbors,
                                       int primary) {
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

extern "C" dn_status dn_fuser_fuse(dn_fuser* f, int64_t* count) {
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
  *count = (int64_t)(f->out_pts.size() / 3);
  return DN_OK;
}

extern "C" dn_status dn_fuser_get(dn_fuser* f, float* points, float* normals, uint8_t* colors,
                                  int64_t capacity) {
  FCHECK(f, "NULL fuser");
  const int64_t n = (int64_t)(f->out_pts.size() / 3);
  FCHECK(capacity >= n, "capacity below the fused point count");
  if (points) std::memcpy(points, f->out_pts.data(), f->out_pts.size() * sizeof(float));
  if (normals) std::memcpy(normals, f->out_nrm.data(), f->out_nrm.size() * sizeof(float));
  if (colors) std::memcpy(colors, f->out_clr.data(), f->out_clr.size());
  return DN_OK;
}
