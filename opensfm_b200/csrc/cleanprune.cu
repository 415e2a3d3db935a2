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
#include "cleanprune.cuh"

namespace dn {
__global__ void __launch_bounds__(256)
clean_kernel(const CleanView* __restrict__ views, int ref, const int* __restrict__ others,
             int n_others, int W, int H, float thr, int min_views, float* __restrict__ out) {
  __shared__ double Kinv[9];
  const CleanView& rv = views[ref];
  if (threadIdx.x == 0 && threadIdx.y == 0) inv3_rn(rv.K, Kinv);
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= H || j >= W) return;
  out[(size_t)i * W + j] = clean_pixel(views, rv, Kinv, others, n_others, i, j, thr, min_views);
}

__global__ void __launch_bounds__(256)
clean_batch_kernel(const CleanView* __restrict__ views, const CleanMap* __restrict__ cmaps,
                   const int* __restrict__ lists, const int4* __restrict__ tiles, float thr,
                   int min_views) {
  clean_tile(views, cmaps, lists, tiles[blockIdx.x], thr, min_views);
}

cudaError_t launch_clean(const CleanView* d_views, int ref, const int* d_others, int n_others,
                         int W, int H, float thr, int min_views, float* out, cudaStream_t s) {
  const dim3 blk(32, 8), grid((W + 31) / 32, (H + 7) / 8);
  clean_kernel<<<grid, blk, 0, s>>>(d_views, ref, d_others, n_others, W, H, thr, min_views, out);
  return cudaGetLastError();
}

cudaError_t launch_clean_batch(const CleanView* d_views, const CleanMap* d_cmaps,
                               const int* d_lists, const int4* d_tiles, int n_tiles, float thr,
                               int min_views, cudaStream_t s) {
  if (n_tiles == 0) return cudaSuccess;
  clean_batch_kernel<<<n_tiles, dim3(kCleanTileX, kCleanTileY), 0, s>>>(d_views, d_cmaps, d_lists,
                                                                         d_tiles, thr, min_views);
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

__global__ void __launch_bounds__(kPruneBlock)
prune_flags_kernel(const PruneView* __restrict__ views, int n_views, float thr,
                   uint8_t* __restrict__ keep, uint32_t* __restrict__ block_counts) {
  prune_flags_block<kPruneBlock>(views, n_views, thr, keep, block_counts, blockIdx.x);
}

__global__ void __launch_bounds__(1024)
scan_counts_kernel(const uint32_t* __restrict__ counts, int n, uint32_t* __restrict__ offsets,
                   unsigned long long* total) {
  scan_counts_block(counts, n, offsets, total);
}

__global__ void __launch_bounds__(kPruneBlock)
prune_write_kernel(const PruneView* __restrict__ views, int n_views, float thr,
                   const uint8_t* __restrict__ keep, const uint32_t* __restrict__ offsets,
                   PruneOut out) {
  prune_write_block<kPruneBlock>(views, n_views, thr, keep, offsets, out, blockIdx.x);
}

// Every map of a batch: tiles (map, block) of kPruneBatchBlock pixels for
// the flags and the writes, one scan block per map.
__global__ void __launch_bounds__(kPruneBatchBlock)
prune_flags_batch_kernel(const PruneMap* __restrict__ pm, const int4* __restrict__ tiles,
                         float thr) {
  const int4 t = tiles[blockIdx.x];
  const PruneMap& m = pm[t.x];
  prune_flags_block<kPruneBatchBlock>(m.views, m.n_views, thr, m.keep, m.counts, t.y);
}

__global__ void __launch_bounds__(1024)
scan_counts_batch_kernel(const PruneMap* __restrict__ pm) {
  const PruneMap& m = pm[blockIdx.x];
  scan_counts_block(m.counts, m.blocks, m.offsets, m.count);
}

__global__ void __launch_bounds__(kPruneBatchBlock)
prune_write_batch_kernel(const PruneMap* __restrict__ pm, const int4* __restrict__ tiles,
                         float thr) {
  const int4 t = tiles[blockIdx.x];
  const PruneMap& m = pm[t.x];
  prune_write_block<kPruneBatchBlock>(m.views, m.n_views, thr, m.keep, m.offsets, m.out, t.y);
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

size_t prune_batch_scratch_bytes(int W, int H) {
  const size_t n = (size_t)W * H;
  const size_t blocks = (n + kPruneBatchBlock - 1) / kPruneBatchBlock;
  const size_t counts = (2 * blocks + 1) * sizeof(uint32_t);
  return ((counts + 255) / 256) * 256 + ((n + 255) / 256) * 256;
}

PruneMap prune_batch_map(const PruneView* d_views, int n_views, int W, int H, void* scratch,
                         PruneOut out, unsigned long long* d_count) {
  const size_t n = (size_t)W * H;
  const int blocks = (int)((n + kPruneBatchBlock - 1) / kPruneBatchBlock);
  const size_t counts_bytes = ((((2 * (size_t)blocks + 1) * sizeof(uint32_t)) + 255) / 256) * 256;
  PruneMap m{};
  m.views = d_views;
  m.n_views = n_views;
  m.blocks = blocks;
  m.counts = static_cast<uint32_t*>(scratch);
  m.offsets = m.counts + blocks;
  m.keep = static_cast<uint8_t*>(scratch) + counts_bytes;
  m.out = out;
  m.count = d_count;
  return m;
}

cudaError_t launch_prune_batch(const PruneMap* d_pm, int n_maps, const int4* d_tiles, int n_tiles,
                               float thr, cudaStream_t s) {
  if (n_maps == 0) return cudaSuccess;
  prune_flags_batch_kernel<<<n_tiles, kPruneBatchBlock, 0, s>>>(d_pm, d_tiles, thr);
  scan_counts_batch_kernel<<<n_maps, 1024, 0, s>>>(d_pm);
  prune_write_batch_kernel<<<n_tiles, kPruneBatchBlock, 0, s>>>(d_pm, d_tiles, thr);
  return cudaGetLastError();
}

}  // namespace dn
