// SVOFuser (svo_fuser.h:14-68, svo_fuser.cc:12-183): TSDF fusion of
// depthmaps into a sparse voxel hash, and surface points at the TSDF's zero
// crossings.
//
// The reference (svo_opencl_kernels.h:187-651) marches every pixel's ray
// through the truncation band, one view per launch, and accumulates
// fixed-point sums into an open-addressing hash keyed by (x, y) in one word
// and z in another, with a "ready" flag between the two writes.  Here:
//   - the voxel key is one 64-bit word (x and y biased to 16 bits, z), so a
//     slot is claimed with a single 64-bit compare-and-swap and needs no
//     ready flag; slots are structure-of-arrays (keys, then nine int32 sums);
//   - all views march in one launch (blockIdx.z is the view): the sums are
//     integer atomic adds, so their order does not matter;
//   - the counting pass uses a key-only table, grown and rerun if a probe
//     sequence ever runs out, so its count is exact;
//   - extraction sorts the occupied voxels (cub radix sort on the key, which
//     orders them by signed x, y, z), finds each voxel's +X, +Y, +Z
//     neighbours in the hash, and compacts the points with a scan, so the
//     output order is ascending voxel order (the reference's follows an
//     atomic counter and is not reproducible) and the reference's cap of a
//     quarter of its table size keeps the first points of that order.
// Arithmetic is FP32 in the order of the kernel source, each operation
// rounded by itself (no contraction), length() as the square root of
// (x*x + y*y) + z*z, division and square root correctly rounded.
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

thread_local std::string g_svo_error;

dn_status sfail(dn_status s, const std::string& m) {
  g_svo_error = m;
  return s;
}

#define SCHECK(cond, msg) \
  do {                    \
    if (!(cond)) return sfail(DN_INVALID_ARG, msg); \
  } while (0)
#define SCUDA(expr)                                                        \
  do {                                                                     \
    cudaError_t e_ = (expr);                                               \
    if (e_ != cudaSuccess) {                                               \
      return sfail(e_ == cudaErrorMemoryAllocation ? DN_OUT_OF_MEMORY      \
                                                   : DN_DEVICE_ERROR,      \
                   cudaGetErrorString(e_));                                \
    }                                                                      \
  } while (0)

typedef unsigned long long u64;
constexpr u64 kEmpty = ~0ull;  // x = 32767 is never stored, so never a key
constexpr int kFpScale = 32768;
constexpr int kWeightScale = 128;
constexpr float kCosThetaMin = 0.15f;
constexpr int kMaxProbes = 256;
constexpr int kFields = 9;  // count, weight, tsdf, nx, ny, nz, r, g, b

struct SvoCam {
  float Kinv[9], Rinv[9], R[9], t[3], cp[3];
};

struct SvoViewDev {
  SvoCam cam;
  int W, H;
  const float* depth;
  const float* normal;   // or null
  const uint8_t* color;  // or null
  const uint8_t* mask;   // or null
  const float* weight;   // or null
};

struct SvoParams {
  float voxel_size, trunc, inv_vs;
  int has_bbox;
  int bmin[3], bmax[3];
};

struct Table {
  u64* keys;
  int* vals;  // [kFields][cap], may be null (counting table)
  u64 cap, mask;
};

// ---------------------------------------------------------------- device
__device__ inline u64 voxel_key(int kx, int ky, int kz) {
  return ((u64)(unsigned)(kx + 32768) << 48) | ((u64)(unsigned)(ky + 32768) << 32) |
         (u64)((unsigned)kz ^ 0x80000000u);
}

__device__ inline u64 key_hash(u64 k) {  // a 64-bit finaliser (multiply-xorshift)
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}

// Claims or finds the key's slot; -1 when kMaxProbes slots are all taken
// by other keys.  *fresh = the slot was claimed by this call.
__device__ inline long long find_or_claim(const Table& t, u64 key, bool* fresh) {
  const u64 h = key_hash(key) & t.mask;
  for (int probe = 0; probe < kMaxProbes; ++probe) {
    const u64 s = (h + (u64)probe) & t.mask;
    const u64 cur = *(volatile u64*)&t.keys[s];
    if (cur == key) {
      *fresh = false;
      return (long long)s;
    }
    if (cur != kEmpty) continue;
    const u64 old = atomicCAS(&t.keys[s], kEmpty, key);
    if (old == kEmpty || old == key) {
      *fresh = old == kEmpty;
      return (long long)s;
    }
  }
  return -1;
}

__device__ inline long long lookup(const Table& t, u64 key) {
  const u64 h = key_hash(key) & t.mask;
  for (int probe = 0; probe < kMaxProbes; ++probe) {
    const u64 s = (h + (u64)probe) & t.mask;
    const u64 cur = t.keys[s];
    if (cur == key) return (long long)s;
    if (cur == kEmpty) return -1;
  }
  return -1;
}

__device__ inline float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ inline float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ inline float fs(float a, float b) { return __fsub_rn(a, b); }

// float -> int as a saturating truncation (NaN -> 0), the GPU's conversion.
__device__ inline int f2i(float x) { return __float2int_rz(x); }

// svo_integrate (counting = false) and svo_count (counting = true) for
// every pixel of every view: x, y pixel; blockIdx.z view.
template <bool COUNTING>
__global__ void svo_march_kernel(const SvoViewDev* __restrict__ views, SvoParams p, Table t,
                                 unsigned* __restrict__ n_unique, int* __restrict__ overflow) {
  const SvoViewDev& v = views[blockIdx.z];
  const int c = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y * blockDim.y + threadIdx.y;
  if (c >= v.W || r >= v.H) return;
  const size_t idx = (size_t)r * v.W + c;
  if (v.mask && v.mask[idx] == 0) return;
  const float d = v.depth[idx];
  if (!(d > 0.0f)) return;
  const SvoCam& cam = v.cam;
  const float uc = (float)c, vr = (float)r;
  const float pc0 = fm(d, fa(fa(fm(cam.Kinv[0], uc), fm(cam.Kinv[1], vr)), cam.Kinv[2]));
  const float pc1 = fm(d, fa(fa(fm(cam.Kinv[3], uc), fm(cam.Kinv[4], vr)), cam.Kinv[5]));
  const float pc2 = fm(d, fa(fa(fm(cam.Kinv[6], uc), fm(cam.Kinv[7], vr)), cam.Kinv[8]));
  const float df0 = fs(pc0, cam.t[0]), df1 = fs(pc1, cam.t[1]), df2 = fs(pc2, cam.t[2]);
  float ray[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const float pw = fa(fa(fm(cam.Rinv[3 * i], df0), fm(cam.Rinv[3 * i + 1], df1)),
                        fm(cam.Rinv[3 * i + 2], df2));
    ray[i] = fs(pw, cam.cp[i]);
  }
  const float ray_len =
      __fsqrt_rn(fa(fa(fm(ray[0], ray[0]), fm(ray[1], ray[1])), fm(ray[2], ray[2])));
  if (ray_len < 1e-8f) return;
  if (fm(ray_len, 1.2e-7f) >= p.voxel_size) return;
#pragma unroll
  for (int i = 0; i < 3; ++i) ray[i] = __fdiv_rn(ray[i], ray_len);
  const float ts = fs(ray_len, p.trunc);
  const float t_start = ts > 0.0f ? ts : 0.0f;
  const float t_end = fa(ray_len, p.trunc);
  int nfp[3] = {0, 0, 0}, rgb[3] = {0, 0, 0}, w_int = 1;
  if (!COUNTING) {
    if (v.normal) {
      const float* nc = v.normal + 3 * idx;
      const float nlen =
          __fsqrt_rn(fa(fa(fm(nc[0], nc[0]), fm(nc[1], nc[1])), fm(nc[2], nc[2])));
      if (nlen > 1e-6f) {
        const float n0 = __fdiv_rn(nc[0], nlen), n1 = __fdiv_rn(nc[1], nlen),
                    n2 = __fdiv_rn(nc[2], nlen);
        float nw[3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
          nw[i] = fa(fa(fm(cam.Rinv[3 * i], n0), fm(cam.Rinv[3 * i + 1], n1)),
                     fm(cam.Rinv[3 * i + 2], n2));
#pragma unroll
        for (int i = 0; i < 3; ++i) nfp[i] = f2i(fm(nw[i], (float)kFpScale));
        const float cs =
            fabsf(fa(fa(fm(ray[0], nw[0]), fm(ray[1], nw[1])), fm(ray[2], nw[2])));
        if (cs < kCosThetaMin) return;  // grazing
      }
    }
    if (v.color)
#pragma unroll
      for (int i = 0; i < 3; ++i) rgb[i] = (int)v.color[3 * idx + i];
    float wf = 1.0f;
    if (v.weight) wf = fm(wf, v.weight[idx]);
    const int wi = f2i(fm(wf, (float)kWeightScale));
    w_int = min(max(wi, 1), 4 * kWeightScale);
  }
  for (float tt = t_start; tt <= t_end; tt = fa(tt, p.voxel_size)) {
    int k[3];
    bool skip = false;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const float s = fa(cam.cp[i], fm(tt, ray[i]));
      const float f = floorf(fm(s, p.inv_vs));
      skip |= !(f >= -2147483648.0f && f < 2147483648.0f);
      k[i] = f2i(f);
    }
    if (skip) continue;
    if (k[0] < -32768 || k[0] > 32766 || k[1] < -32768 || k[1] > 32766) continue;
    if (p.has_bbox && (k[0] < p.bmin[0] || k[0] > p.bmax[0] || k[1] < p.bmin[1] ||
                       k[1] > p.bmax[1] || k[2] < p.bmin[2] || k[2] > p.bmax[2]))
      continue;
    const float c0 = fm(fa((float)k[0], 0.5f), p.voxel_size);
    const float c1 = fm(fa((float)k[1], 0.5f), p.voxel_size);
    const float c2 = fm(fa((float)k[2], 0.5f), p.voxel_size);
    const float zc = fa(fa(fa(fm(cam.R[6], c0), fm(cam.R[7], c1)), fm(cam.R[8], c2)), cam.t[2]);
    if (zc <= 0.0f) continue;
    const float sdf = fs(d, zc);
    if (sdf < -p.trunc) continue;
    const u64 key = voxel_key(k[0], k[1], k[2]);
    bool fresh = false;
    const long long s = find_or_claim(t, key, &fresh);
    if (s < 0) {
      atomicExch(overflow, 1);
      continue;
    }
    if (COUNTING) {
      if (fresh) atomicAdd(n_unique, 1u);
      continue;
    }
    const float q = __fdiv_rn(sdf, p.trunc);
    const float tsdf = q < 1.0f ? q : 1.0f;
    const int tfp = f2i(fm(tsdf, (float)kFpScale));
    int* vals = t.vals;
    const u64 C = t.cap;
    atomicAdd(&vals[0 * C + s], 1);
    atomicAdd(&vals[1 * C + s], w_int);
    atomicAdd(&vals[2 * C + s], tfp * w_int);
    atomicAdd(&vals[3 * C + s], nfp[0] * w_int);
    atomicAdd(&vals[4 * C + s], nfp[1] * w_int);
    atomicAdd(&vals[5 * C + s], nfp[2] * w_int);
    atomicAdd(&vals[6 * C + s], rgb[0] * w_int);
    atomicAdd(&vals[7 * C + s], rgb[1] * w_int);
    atomicAdd(&vals[8 * C + s], rgb[2] * w_int);
  }
}

// Occupied slots as (key, slot) for the sort.
__global__ void svo_occupied_kernel(Table t, u64* __restrict__ okey, unsigned* __restrict__ oslot,
                                    unsigned* __restrict__ n_occ) {
  const u64 s = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= t.cap) return;
  const u64 k = t.keys[s];
  if (k == kEmpty || t.vals[s] == 0) return;  // count 0: skipped by the extraction
  const unsigned o = atomicAdd(n_occ, 1u);
  okey[o] = k;
  oslot[o] = (unsigned)s;
}

__device__ inline float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// svo_extract_points (svo_opencl_kernels.h:546-651) for the i-th voxel in
// key order: up to three points at out[3 i + axis], flag[3 i + axis].
__global__ void svo_extract_kernel(Table t, const u64* __restrict__ skey,
                                   const unsigned* __restrict__ sslot, unsigned n_occ, float mws,
                                   float vs, float* __restrict__ tp, float* __restrict__ tn,
                                   uint8_t* __restrict__ tc, unsigned* __restrict__ flag) {
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_occ) return;
  for (int d = 0; d < 3; ++d) flag[3 * i + d] = 0;
  const u64 a = sslot[i];
  const u64 C = t.cap;
  const float sw_a = (float)t.vals[1 * C + a];
  if (sw_a < mws) return;
  const u64 ka = skey[i];
  const int kx = (int)((ka >> 48) & 0xFFFF) - 32768;
  const int ky = (int)((ka >> 32) & 0xFFFF) - 32768;
  const int kz = (int)((unsigned)ka ^ 0x80000000u);
  const float inv_sw_a = __fdiv_rn(1.0f, sw_a);
  const float inv_fp_sw_a = __fdiv_rn(inv_sw_a, (float)kFpScale);
  const float tsdf_a = fm((float)t.vals[2 * C + a], inv_fp_sw_a);
  float na[3], ca[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    na[j] = fm((float)t.vals[(3 + j) * C + a], inv_fp_sw_a);
    ca[j] = fm((float)t.vals[(6 + j) * C + a], inv_sw_a);
  }
  for (int d = 0; d < 3; ++d) {
    const int nb[3] = {kx + (d == 0), ky + (d == 1), kz + (d == 2)};
    if (nb[0] > 32766 || nb[1] > 32766) continue;  // never stored
    const long long b = lookup(t, voxel_key(nb[0], nb[1], nb[2]));
    if (b < 0) continue;
    const float sw_b = (float)t.vals[1 * C + b];
    if (sw_b < mws) continue;
    const float inv_sw_b = __fdiv_rn(1.0f, sw_b);
    const float inv_fp_sw_b = __fdiv_rn(inv_sw_b, (float)kFpScale);
    const float tsdf_b = fm((float)t.vals[2 * C + b], inv_fp_sw_b);
    if ((tsdf_a > 0.0f) == (tsdf_b > 0.0f)) continue;
    if (tsdf_a == 0.0f || tsdf_b == 0.0f) continue;
    const float tt = clampf(__fdiv_rn(tsdf_a, fs(tsdf_a, tsdf_b)), 0.0f, 1.0f);
    const int kav[3] = {kx, ky, kz};
    float nn[3];
    const size_t o = 3 * (size_t)i + d;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float pa = fm(fa((float)kav[j], 0.5f), vs);
      const float pb = fm(fa((float)nb[j], 0.5f), vs);
      tp[3 * o + j] = fa(pa, fm(tt, fs(pb, pa)));
      const float nbj = fm((float)t.vals[(3 + j) * C + b], inv_fp_sw_b);
      nn[j] = fa(na[j], fm(tt, fs(nbj, na[j])));
    }
    const float nlen =
        __fsqrt_rn(fa(fa(fm(nn[0], nn[0]), fm(nn[1], nn[1])), fm(nn[2], nn[2])));
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      tn[3 * o + j] = nlen > 1e-6f ? __fdiv_rn(nn[j], nlen) : nn[j];
      const float cbj = fm((float)t.vals[(6 + j) * C + b], inv_sw_b);
      tc[3 * o + j] = (uint8_t)f2i(clampf(fa(ca[j], fm(tt, fs(cbj, ca[j]))), 0.0f, 255.0f));
    }
    flag[o] = 1;
  }
}

__global__ void svo_scatter_kernel(const float* __restrict__ tp, const float* __restrict__ tn,
                                   const uint8_t* __restrict__ tc,
                                   const unsigned* __restrict__ flag,
                                   const unsigned* __restrict__ pos, size_t n_slots,
                                   unsigned max_out, float* __restrict__ op,
                                   float* __restrict__ on, uint8_t* __restrict__ oc) {
  const size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n_slots || !flag[o]) return;
  const unsigned q = pos[o];
  if (q >= max_out) return;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    op[3 * (size_t)q + j] = tp[3 * o + j];
    on[3 * (size_t)q + j] = tn[3 * o + j];
    oc[3 * (size_t)q + j] = tc[3 * o + j];
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

// Eigen's 3x3 inverse: cofactors, determinant from the first column.
void inv3(const float* m, float* o) {
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

struct SView {
  SvoCam cam;
  int W = 0, H = 0;
  DBuf<float> depth, normal, weight;
  DBuf<uint8_t> color, mask;
  bool has_normal = false, has_color = false, has_mask = false, has_weight = false;
};

u64 pow2_at_least(u64 v) {
  u64 c = 1;
  while (c < v) c <<= 1;
  return c;
}

}  // namespace

struct dn_svo {
  int device = 0;
  cudaStream_t stream = nullptr;
  float voxel_size = 0.02f, trunc_factor = 4.0f, min_weight = 3.0f;  // svo_fuser.cc:12-13
  bool has_bbox = false;
  float bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
  std::vector<std::unique_ptr<SView>> views;
  uint32_t last_count = 0;
  std::vector<float> out_pts, out_nrm;
  std::vector<uint8_t> out_clr;
  float fuse_ms = 0.0f;
  ~dn_svo() {
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

SvoParams make_params(const dn_svo* f) {
  SvoParams p;
  p.voxel_size = f->voxel_size;
  p.trunc = f->trunc_factor * f->voxel_size;
  p.inv_vs = 1.0f / f->voxel_size;
  p.has_bbox = f->has_bbox ? 1 : 0;
  for (int i = 0; i < 3; ++i) {
    // svo_fuser.cc:62-66: floor / ceil of the corners in voxel units.
    p.bmin[i] = f->has_bbox ? (int)std::floor(f->bmin[i] * p.inv_vs) : 0;
    p.bmax[i] = f->has_bbox ? (int)std::ceil(f->bmax[i] * p.inv_vs) : 0;
  }
  return p;
}

dn_status upload_views(dn_svo* f, DBuf<SvoViewDev>& d_views, int* max_w, int* max_h) {
  const int nv = (int)f->views.size();
  std::vector<SvoViewDev> hv(nv);
  *max_w = *max_h = 0;
  for (int i = 0; i < nv; ++i) {
    const SView& v = *f->views[i];
    hv[i].cam = v.cam;
    hv[i].W = v.W;
    hv[i].H = v.H;
    hv[i].depth = v.depth.p;
    hv[i].normal = v.has_normal ? v.normal.p : nullptr;
    hv[i].color = v.has_color ? v.color.p : nullptr;
    hv[i].mask = v.has_mask ? v.mask.p : nullptr;
    hv[i].weight = v.has_weight ? v.weight.p : nullptr;
    *max_w = std::max(*max_w, v.W);
    *max_h = std::max(*max_h, v.H);
  }
  SCUDA(d_views.alloc(nv));
  SCUDA(cudaMemcpyAsync(d_views.p, hv.data(), nv * sizeof(SvoViewDev), cudaMemcpyHostToDevice,
                        f->stream));
  return DN_OK;
}

}  // namespace

extern "C" const char* dn_svo_last_error(void) { return g_svo_error.c_str(); }

extern "C" dn_status dn_svo_create(dn_svo** out) {
  const dn::DeviceRestore device_restore_;
  SCHECK(out, "NULL output");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return sfail(DN_DEVICE_ERROR, "no CUDA device");
  auto f = std::make_unique<dn_svo>();
  SCUDA(cudaGetDevice(&f->device));
  SCUDA(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking));
  *out = f.release();
  return DN_OK;
}
extern "C" dn_status dn_svo_destroy(dn_svo* f) {
  const dn::DeviceRestore device_restore_;
  if (f) cudaSetDevice(f->device);
  delete f;
  return DN_OK;
}
extern "C" dn_status dn_svo_set_voxel_size(dn_svo* f, float size) {
  const dn::DeviceRestore device_restore_;
  SCHECK(f, "NULL fuser");
  f->voxel_size = std::max(1e-6f, size);  // svo_fuser.cc:15
  return DN_OK;
}
extern "C" dn_status dn_svo_set_trunc_factor(dn_svo* f, float factor) {
  const dn::DeviceRestore device_restore_;
  SCHECK(f, "NULL fuser");
  f->trunc_factor = std::max(1.0f, factor);  // svo_fuser.cc:17-19
  return DN_OK;
}
extern "C" dn_status dn_svo_set_min_weight(dn_svo* f, float w) {
  const dn::DeviceRestore device_restore_;
  SCHECK(f, "NULL fuser");
  f->min_weight = std::max(0.0f, w);  // svo_fuser.cc:21
  return DN_OK;
}
extern "C" dn_status dn_svo_set_device(dn_svo* f, int device) {
  const dn::DeviceRestore device_restore_;
  SCHECK(f, "NULL fuser");
  SCHECK(f->views.empty(), "set_device must come before add_view");
  int n = 0;
  SCUDA(cudaGetDeviceCount(&n));
  SCHECK(device >= 0 && device < n, "no such CUDA device");
  SCUDA(cudaSetDevice(device));
  cudaStream_t s;
  SCUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  cudaSetDevice(f->device);
  cudaStreamDestroy(f->stream);
  f->stream = s;
  f->device = device;
  return DN_OK;
}
extern "C" dn_status dn_svo_set_bbox(dn_svo* f, const float min_world[3],
                                     const float max_world[3]) {
  const dn::DeviceRestore device_restore_;
  SCHECK(f && min_world && max_world, "NULL argument");
  f->has_bbox = true;
  for (int i = 0; i < 3; ++i) {
    f->bmin[i] = min_world[i];
    f->bmax[i] = max_world[i];
  }
  return DN_OK;
}

extern "C" dn_status dn_svo_add_view(dn_svo* f, const double* K, const double* R,
                                     const double* t, const float* depth, const float* normal,
                                     const uint8_t* color, const uint8_t* mask,
                                     const float* weight, int width, int height) {
  const dn::DeviceRestore device_restore_;
  SCHECK(f, "NULL fuser");
  SCHECK(K && R && t && depth, "NULL argument");
  SCHECK(width >= 1 && height >= 1 && width <= 16384 && height <= 16384, "bad depthmap size");
  for (int i = 0; i < 9; ++i) SCHECK(std::isfinite(K[i]) && std::isfinite(R[i]), "K, R must be finite");
  for (int i = 0; i < 3; ++i) SCHECK(std::isfinite(t[i]), "t must be finite");
  SCUDA(cudaSetDevice(f->device));
  auto v = std::make_unique<SView>();
  // svo_opencl.cc:213-226 over the float casts of K, R, t.
  float Kf[9];
  for (int i = 0; i < 9; ++i) {
    Kf[i] = (float)K[i];
    v->cam.R[i] = (float)R[i];
  }
  for (int i = 0; i < 3; ++i) v->cam.t[i] = (float)t[i];
  inv3(Kf, v->cam.Kinv);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) v->cam.Rinv[3 * i + j] = v->cam.R[3 * j + i];
  for (int i = 0; i < 3; ++i)
    v->cam.cp[i] = ((-v->cam.Rinv[3 * i] * v->cam.t[0]) + (-v->cam.Rinv[3 * i + 1] * v->cam.t[1])) +
                   (-v->cam.Rinv[3 * i + 2] * v->cam.t[2]);
  v->W = width;
  v->H = height;
  const size_t npx = (size_t)width * height;
  SCUDA(v->depth.alloc(npx));
  SCUDA(cudaMemcpyAsync(v->depth.p, depth, npx * sizeof(float), cudaMemcpyHostToDevice, f->stream));
  if (normal) {
    v->has_normal = true;
    SCUDA(v->normal.alloc(3 * npx));
    SCUDA(cudaMemcpyAsync(v->normal.p, normal, 3 * npx * sizeof(float), cudaMemcpyHostToDevice,
                          f->stream));
  }
  if (color) {
    v->has_color = true;
    SCUDA(v->color.alloc(3 * npx));
    SCUDA(cudaMemcpyAsync(v->color.p, color, 3 * npx, cudaMemcpyHostToDevice, f->stream));
  }
  if (mask) {
    v->has_mask = true;
    SCUDA(v->mask.alloc(npx));
    SCUDA(cudaMemcpyAsync(v->mask.p, mask, npx, cudaMemcpyHostToDevice, f->stream));
  }
  if (weight) {
    v->has_weight = true;
    SCUDA(v->weight.alloc(npx));
    SCUDA(cudaMemcpyAsync(v->weight.p, weight, npx * sizeof(float), cudaMemcpyHostToDevice,
                          f->stream));
  }
  SCUDA(cudaStreamSynchronize(f->stream));
  f->views.push_back(std::move(v));
  return DN_OK;
}

// The march over every view into table `t`; *overflow set if a probe
// sequence ran out.
static dn_status march(dn_svo* f, bool counting, const DBuf<SvoViewDev>& d_views, int max_w,
                       int max_h, const Table& t, unsigned* d_unique, int* d_overflow) {
  const SvoParams p = make_params(f);
  const dim3 blk(32, 8), grid((max_w + 31) / 32, (max_h + 7) / 8, (unsigned)f->views.size());
  if (counting)
    svo_march_kernel<true><<<grid, blk, 0, f->stream>>>(d_views.p, p, t, d_unique, d_overflow);
  else
    svo_march_kernel<false><<<grid, blk, 0, f->stream>>>(d_views.p, p, t, d_unique, d_overflow);
  SCUDA(cudaGetLastError());
  return DN_OK;
}

extern "C" dn_status dn_svo_count_voxels(dn_svo* f, uint32_t* count) {
  const dn::DeviceRestore device_restore_;
  SCHECK(f && count, "NULL argument");
  *count = 0;
  if (f->views.empty()) return DN_OK;  // svo_fuser.cc:53-55
  SCUDA(cudaSetDevice(f->device));
  DBuf<SvoViewDev> d_views;
  int mw = 0, mh = 0;
  dn_status st = upload_views(f, d_views, &mw, &mh);
  if (st != DN_OK) return st;
  // Table sized from the reference's estimate (svo_fuser.cc:80-89), doubled
  // for a half-full table; grown and rerun if a probe sequence runs out.
  uint64_t max_px = 0;
  for (auto& v : f->views) max_px = std::max<uint64_t>(max_px, (uint64_t)v->W * v->H);
  const double est = (double)max_px * std::ceil(4.0 * f->trunc_factor) *
                     std::sqrt((double)f->views.size());
  u64 cap = pow2_at_least(std::min<u64>(std::max<u64>((u64)std::min(est, 1e10) * 2, 1u << 20),
                                         1ull << 29));
  DBuf<u64> keys;
  DBuf<unsigned> d_unique;
  DBuf<int> d_overflow;
  SCUDA(d_unique.alloc(1));
  SCUDA(d_overflow.alloc(1));
  for (int attempt = 0; attempt < 8; ++attempt) {
    SCUDA(keys.alloc(cap));
    SCUDA(cudaMemsetAsync(keys.p, 0xFF, cap * sizeof(u64), f->stream));
    SCUDA(cudaMemsetAsync(d_unique.p, 0, sizeof(unsigned), f->stream));
    SCUDA(cudaMemsetAsync(d_overflow.p, 0, sizeof(int), f->stream));
    Table t{keys.p, nullptr, cap, cap - 1};
    st = march(f, true, d_views, mw, mh, t, d_unique.p, d_overflow.p);
    if (st != DN_OK) return st;
    unsigned n = 0;
    int ovf = 0;
    SCUDA(cudaMemcpyAsync(&n, d_unique.p, sizeof(unsigned), cudaMemcpyDeviceToHost, f->stream));
    SCUDA(cudaMemcpyAsync(&ovf, d_overflow.p, sizeof(int), cudaMemcpyDeviceToHost, f->stream));
    SCUDA(cudaStreamSynchronize(f->stream));
    if (!ovf) {
      *count = n;
      f->last_count = n;
      return DN_OK;
    }
    keys.release();
    cap *= 2;
  }
  return sfail(DN_OUT_OF_MEMORY, "voxel counting table kept overflowing");
}

extern "C" dn_status dn_svo_fuse(dn_svo* f, int64_t* count) {
  const dn::DeviceRestore device_restore_;
  SCHECK(f && count, "NULL argument");
  *count = 0;
  f->out_pts.clear();
  f->out_nrm.clear();
  f->out_clr.clear();
  f->fuse_ms = 0.0f;
  if (f->views.empty()) return DN_OK;  // svo_fuser.cc:118-120
  SCHECK(f->last_count != 0, "CountVoxels() must be called before Fuse()");  // :122-125
  SCUDA(cudaSetDevice(f->device));
  cudaEvent_t e0, e1;
  SCUDA(cudaEventCreate(&e0));
  SCUDA(cudaEventCreate(&e1));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } evg{e0, e1};
  DBuf<SvoViewDev> d_views;
  int mw = 0, mh = 0;
  dn_status st = upload_views(f, d_views, &mw, &mh);
  if (st != DN_OK) return st;
  // The reference's table: max(2 count, 2^20) slots rounded up to a power
  // of two (svo_fuser.cc:139-142, svo_opencl.cc:61-65); it emits at most a
  // quarter of that (svo_opencl.cc:549).
  const u64 ref_cap = pow2_at_least(std::max<u64>((u64)f->last_count * 2, 1u << 20));
  const unsigned max_out = (unsigned)std::min<u64>(ref_cap / 4, 0xFFFFFFFFu);
  u64 cap = ref_cap;
  DBuf<u64> keys;
  DBuf<int> vals;
  DBuf<unsigned> d_n;
  DBuf<int> d_overflow;
  SCUDA(d_n.alloc(1));
  SCUDA(d_overflow.alloc(1));
  SCUDA(cudaEventRecord(e0, f->stream));
  Table t{};
  for (int attempt = 0;; ++attempt) {
    if (attempt == 8) return sfail(DN_OUT_OF_MEMORY, "voxel table kept overflowing");
    SCUDA(keys.alloc(cap));
    SCUDA(vals.alloc(kFields * cap));
    SCUDA(cudaMemsetAsync(keys.p, 0xFF, cap * sizeof(u64), f->stream));
    SCUDA(cudaMemsetAsync(vals.p, 0, kFields * cap * sizeof(int), f->stream));
    SCUDA(cudaMemsetAsync(d_overflow.p, 0, sizeof(int), f->stream));
    t = Table{keys.p, vals.p, cap, cap - 1};
    st = march(f, false, d_views, mw, mh, t, d_n.p, d_overflow.p);
    if (st != DN_OK) return st;
    int ovf = 0;
    SCUDA(cudaMemcpyAsync(&ovf, d_overflow.p, sizeof(int), cudaMemcpyDeviceToHost, f->stream));
    SCUDA(cudaStreamSynchronize(f->stream));
    if (!ovf) break;
    keys.release();
    vals.release();
    cap *= 2;
  }
  // Occupied voxels in key order.
  DBuf<u64> okey, skey;
  DBuf<unsigned> oslot, sslot;
  SCUDA(okey.alloc(cap));
  SCUDA(oslot.alloc(cap));
  SCUDA(cudaMemsetAsync(d_n.p, 0, sizeof(unsigned), f->stream));
  svo_occupied_kernel<<<(unsigned)((cap + 255) / 256), 256, 0, f->stream>>>(t, okey.p, oslot.p,
                                                                             d_n.p);
  SCUDA(cudaGetLastError());
  unsigned n_occ = 0;
  SCUDA(cudaMemcpyAsync(&n_occ, d_n.p, sizeof(unsigned), cudaMemcpyDeviceToHost, f->stream));
  SCUDA(cudaStreamSynchronize(f->stream));
  unsigned n_pts = 0;
  DBuf<float> op, on;
  DBuf<uint8_t> oc;
  if (n_occ) {
    SCUDA(skey.alloc(n_occ));
    SCUDA(sslot.alloc(n_occ));
    DBuf<uint8_t> tmp;
    size_t tb = 0;
    SCUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, okey.p, skey.p, oslot.p, sslot.p,
                                          (int)n_occ, 0, 64, f->stream));
    SCUDA(tmp.alloc(std::max<size_t>(tb, 1)));
    SCUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, okey.p, skey.p, oslot.p, sslot.p,
                                          (int)n_occ, 0, 64, f->stream));
    const size_t n_slots = 3 * (size_t)n_occ;
    DBuf<float> tp, tn;
    DBuf<uint8_t> tc;
    DBuf<unsigned> flag, pos;
    SCUDA(tp.alloc(3 * n_slots));
    SCUDA(tn.alloc(3 * n_slots));
    SCUDA(tc.alloc(3 * n_slots));
    SCUDA(flag.alloc(n_slots));
    SCUDA(pos.alloc(n_slots));
    const float mws = f->min_weight * (float)kWeightScale;
    svo_extract_kernel<<<(n_occ + 127) / 128, 128, 0, f->stream>>>(
        t, skey.p, sslot.p, n_occ, mws, f->voxel_size, tp.p, tn.p, tc.p, flag.p);
    SCUDA(cudaGetLastError());
    SCUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag.p, pos.p, (int)n_slots, f->stream));
    SCUDA(tmp.alloc(std::max<size_t>(tb, 1)));
    SCUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, flag.p, pos.p, (int)n_slots, f->stream));
    unsigned last[2] = {0, 0};
    SCUDA(cudaMemcpyAsync(&last[0], pos.p + n_slots - 1, sizeof(unsigned), cudaMemcpyDeviceToHost,
                          f->stream));
    SCUDA(cudaMemcpyAsync(&last[1], flag.p + n_slots - 1, sizeof(unsigned),
                          cudaMemcpyDeviceToHost, f->stream));
    SCUDA(cudaStreamSynchronize(f->stream));
    n_pts = std::min(last[0] + last[1], max_out);
    if (n_pts) {
      SCUDA(op.alloc(3 * (size_t)n_pts));
      SCUDA(on.alloc(3 * (size_t)n_pts));
      SCUDA(oc.alloc(3 * (size_t)n_pts));
      svo_scatter_kernel<<<(unsigned)((n_slots + 255) / 256), 256, 0, f->stream>>>(
          tp.p, tn.p, tc.p, flag.p, pos.p, n_slots, n_pts, op.p, on.p, oc.p);
      SCUDA(cudaGetLastError());
    }
    SCUDA(cudaEventRecord(e1, f->stream));
    f->out_pts.resize(3 * (size_t)n_pts);
    f->out_nrm.resize(3 * (size_t)n_pts);
    f->out_clr.resize(3 * (size_t)n_pts);
    if (n_pts) {
      SCUDA(cudaMemcpyAsync(f->out_pts.data(), op.p, 3 * (size_t)n_pts * sizeof(float),
                            cudaMemcpyDeviceToHost, f->stream));
      SCUDA(cudaMemcpyAsync(f->out_nrm.data(), on.p, 3 * (size_t)n_pts * sizeof(float),
                            cudaMemcpyDeviceToHost, f->stream));
      SCUDA(cudaMemcpyAsync(f->out_clr.data(), oc.p, 3 * (size_t)n_pts, cudaMemcpyDeviceToHost,
                            f->stream));
    }
    SCUDA(cudaStreamSynchronize(f->stream));
  } else {
    SCUDA(cudaEventRecord(e1, f->stream));
    SCUDA(cudaStreamSynchronize(f->stream));
  }
  SCUDA(cudaEventElapsedTime(&f->fuse_ms, e0, e1));
  *count = n_pts;
  return DN_OK;
}

extern "C" dn_status dn_svo_get(dn_svo* f, float* points, float* normals, uint8_t* colors,
                                int64_t capacity) {
  const dn::DeviceRestore device_restore_;
  SCHECK(f, "NULL fuser");
  const int64_t n = (int64_t)(f->out_pts.size() / 3);
  SCHECK(capacity >= n, "capacity below the fused point count");
  if (points) std::memcpy(points, f->out_pts.data(), f->out_pts.size() * sizeof(float));
  if (normals) std::memcpy(normals, f->out_nrm.data(), f->out_nrm.size() * sizeof(float));
  if (colors) std::memcpy(colors, f->out_clr.data(), f->out_clr.size());
  return DN_OK;
}

extern "C" dn_status dn_svo_last_fuse_ms(dn_svo* f, float* ms) {
  const dn::DeviceRestore device_restore_;
  SCHECK(f && ms, "NULL argument");
  *ms = f->fuse_ms;
  return DN_OK;
}
