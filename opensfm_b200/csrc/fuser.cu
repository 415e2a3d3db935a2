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
                                       float* __restrict__ cand_pt, float* __restrict__ cand_nrm) {
  const ViewDevF& ref = views[ri];
  const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y * blockDim.y + threadIdx.y;
  if (c >= ref.W || r >= ref.H) return;
  const size_t rp = (size_t)r * ref.W + c;
  const int bm = p.border;
  bool ok = r >= bm && r < ref.H - bm && c >= bm && c < ref.W - bm;
  ok = ok && !(ref.mask && ref.mask[rp] == 0);
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
            if (!(src.mask && src.mask[sp] == 0)) {
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
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      cand_pt[3 * slot + d] = spt[d];
      cand_nrm[3 * slot + d] = snw[d];
    }
  }
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
  std::vector<uint8_t> color;  // [H][W][3], host: colours are read by the host pass
  std::vector<int> nbrs;
  bool primary = true;
  bool has_mask = false;
  DBuf<float> depth, normal;
  DBuf<uint8_t> mask;
};

template <typename T>
T nth_median(T* v, int n) {
  std::nth_element(v, v + n / 2, v + n);
  return v[n / 2];
}

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
  v->color.assign(color, color + 3 * npx);
  v->nbrs.assign(neighbor_ids, neighbor_ids + n_neighbors);
  v->primary = primary != 0;
  FCUDA(v->depth.alloc(npx));
  FCUDA(v->normal.alloc(3 * npx));
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
  }
  DBuf<ViewDevF> d_views;
  FCUDA(d_views.alloc(nv));
  FCUDA(cudaMemcpyAsync(d_views.p, hv.data(), nv * sizeof(ViewDevF), cudaMemcpyHostToDevice,
                        f->stream));
  Params p;
  p.max_reproj_sq = f->max_reproj_error_sq;
  p.max_depth_error = f->max_depth_error;
  p.min_cos = std::cos(f->max_normal_deg * static_cast<float>(M_PI) / 180.0f);
  p.behind = f->behind;
  p.border = f->border;

  std::vector<std::vector<uint8_t>> fused(nv);
  for (int i = 0; i < nv; ++i) fused[i].assign((size_t)f->views[i]->W * f->views[i]->H, 0);
  DBuf<int> d_nbrs;
  DBuf<uint8_t> d_ok;
  DBuf<float> d_rpt, d_rnrm, d_cpt, d_cnrm;
  DBuf<int> d_cpix;
  HBuf<uint8_t> h_ok;
  HBuf<float> h_rpt, h_rnrm, h_cpt, h_cnrm;
  HBuf<int> h_cpix;
  int max_obs = 1;
  for (int i = 0; i < nv; ++i) max_obs = std::max(max_obs, 1 + (int)f->views[i]->nbrs.size());
  std::vector<float> comp(max_obs), pts(3 * max_obs), nrm(3 * max_obs);
  std::vector<uint8_t> comp8(max_obs), clr(3 * max_obs);
  std::vector<int> used_v(max_obs), used_p(max_obs);

  for (int ri = 0; ri < nv; ++ri) {
    const FView& ref = *f->views[ri];
    if (!ref.primary) continue;
    const int nn = (int)ref.nbrs.size();
    const size_t npx = (size_t)ref.W * ref.H;
    const size_t nslot = npx * (size_t)std::max(nn, 1);
    FCUDA(d_nbrs.alloc(std::max(nn, 1)));
    if (nn)
      FCUDA(cudaMemcpyAsync(d_nbrs.p, ref.nbrs.data(), nn * sizeof(int), cudaMemcpyHostToDevice,
                            f->stream));
    FCUDA(d_ok.alloc(npx));
    FCUDA(d_rpt.alloc(3 * npx));
    FCUDA(d_rnrm.alloc(3 * npx));
    FCUDA(d_cpix.alloc(nslot));
    FCUDA(d_cpt.alloc(3 * nslot));
    FCUDA(d_cnrm.alloc(3 * nslot));
    const dim3 blk(32, 8), grid((ref.W + 31) / 32, (ref.H + 7) / 8);
    fuse_candidates_kernel<<<grid, blk, 0, f->stream>>>(d_views.p, nv, ri, d_nbrs.p, nn, p,
                                                        d_ok.p, d_rpt.p, d_rnrm.p, d_cpix.p,
                                                        d_cpt.p, d_cnrm.p);
    FCUDA(cudaGetLastError());
    FCUDA(h_ok.alloc(npx));
    FCUDA(h_rpt.alloc(3 * npx));
    FCUDA(h_rnrm.alloc(3 * npx));
    FCUDA(h_cpix.alloc(nslot));
    FCUDA(h_cpt.alloc(3 * nslot));
    FCUDA(h_cnrm.alloc(3 * nslot));
    FCUDA(cudaMemcpyAsync(h_ok.p, d_ok.p, npx, cudaMemcpyDeviceToHost, f->stream));
    FCUDA(cudaMemcpyAsync(h_rpt.p, d_rpt.p, 3 * npx * sizeof(float), cudaMemcpyDeviceToHost,
                          f->stream));
    FCUDA(cudaMemcpyAsync(h_rnrm.p, d_rnrm.p, 3 * npx * sizeof(float), cudaMemcpyDeviceToHost,
                          f->stream));
    if (nn) {
      FCUDA(cudaMemcpyAsync(h_cpix.p, d_cpix.p, npx * nn * sizeof(int), cudaMemcpyDeviceToHost,
                            f->stream));
      FCUDA(cudaMemcpyAsync(h_cpt.p, d_cpt.p, 3 * npx * nn * sizeof(float),
                            cudaMemcpyDeviceToHost, f->stream));
      FCUDA(cudaMemcpyAsync(h_cnrm.p, d_cnrm.p, 3 * npx * nn * sizeof(float),
                            cudaMemcpyDeviceToHost, f->stream));
    }
    FCUDA(cudaStreamSynchronize(f->stream));

    // The reference's raster walk: marks, then medians (fuser.cc:163-355).
    std::vector<uint8_t>& rf = fused[ri];
    for (size_t rp = 0; rp < npx; ++rp) {
      if (rf[rp] || !h_ok.p[rp]) continue;
      int n_obs = 1, n_used = 0;
      for (int d = 0; d < 3; ++d) {
        pts[d] = h_rpt.p[3 * rp + d];
        nrm[d] = h_rnrm.p[3 * rp + d];
        clr[d] = ref.color[3 * rp + d];
      }
      for (int k = 0; k < nn; ++k) {
        const size_t slot = rp * nn + k;
        const int sp = h_cpix.p[slot];
        if (sp < 0) continue;
        const int si = ref.nbrs[k];
        if (fused[si][sp]) continue;
        for (int d = 0; d < 3; ++d) {
          pts[3 * n_obs + d] = h_cpt.p[3 * slot + d];
          nrm[3 * n_obs + d] = h_cnrm.p[3 * slot + d];
          clr[3 * n_obs + d] = f->views[si]->color[3 * (size_t)sp + d];
        }
        ++n_obs;
        used_v[n_used] = si;
        used_p[n_used] = sp;
        ++n_used;
      }
      if (n_obs < f->min_num_consistent) continue;
      float mp[3], mn[3];
      uint8_t mc[3];
      for (int d = 0; d < 3; ++d) {
        for (int k = 0; k < n_obs; ++k) comp[k] = pts[3 * k + d];
        mp[d] = nth_median(comp.data(), n_obs);
      }
      for (int d = 0; d < 3; ++d) {
        for (int k = 0; k < n_obs; ++k) comp[k] = nrm[3 * k + d];
        mn[d] = nth_median(comp.data(), n_obs);
      }
      const float ml = std::sqrt((mn[0] * mn[0] + mn[1] * mn[1]) + mn[2] * mn[2]);
      if (ml > 1e-6f)
        for (int d = 0; d < 3; ++d) mn[d] = mn[d] / ml;
      for (int d = 0; d < 3; ++d) {
        for (int k = 0; k < n_obs; ++k) comp8[k] = clr[3 * k + d];
        mc[d] = nth_median(comp8.data(), n_obs);
      }
      f->out_pts.insert(f->out_pts.end(), mp, mp + 3);
      f->out_nrm.insert(f->out_nrm.end(), mn, mn + 3);
      f->out_clr.insert(f->out_clr.end(), mc, mc + 3);
      rf[rp] = 1;
      for (int k = 0; k < n_used; ++k) fused[used_v[k]][used_p[k]] = 1;
    }
  }
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
