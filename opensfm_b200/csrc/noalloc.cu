// DepthmapPruner::Prune without any device allocation (dn_prune_noalloc).
//
// The regular pruner (dn_pruner_*) allocates its working buffers with
// cudaMalloc.  Some callers cannot: a host application that hands the whole
// GPU to its own memory pool (for example a framework that reserves most of
// device memory at start-up), or code that must not allocate once it is
// running (a real-time loop, a process with a fixed memory budget).  This
// entry point takes device inputs and device outputs from the caller and
// keeps its own working memory in the file-scope arrays below, which exist
// once per GPU for the life of the process.
//
// Limits and sharing:
//  - at most kNoAllocMaxPixels (4,194,304, e.g. 2048 x 2048) pixels in the
//    reference depthmap and kNoAllocMaxViews (17) views; larger requests are
//    rejected with DN_INVALID_ARG;
//  - every call uses the same arrays, which keep the previous call's
//    contents (each call overwrites all it reads, so nothing needs clearing);
//    calls whose GPU work overlaps (on different streams, or from different
//    host threads) race on them and must be serialised by the caller;
//  - the first call on a device looks up the arrays' device addresses
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture on the device.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "dense_b200.h"
#include "kernels.h"

namespace {

constexpr long long kNoAllocMaxPixels = 4LL * 1024 * 1024;
constexpr int kNoAllocMaxViews = 17;
// Keep flags (1 byte per pixel) plus per-256-pixel block counts and offsets,
// each rounded up to 256 bytes (matches dn::prune_scratch_bytes).
constexpr size_t kNoAllocBlocks = (size_t)(kNoAllocMaxPixels + 255) / 256;
constexpr size_t kNoAllocScratchBytes =
    (((2 * kNoAllocBlocks + 1) * sizeof(uint32_t) + 255) / 256) * 256 +
    (((size_t)kNoAllocMaxPixels + 255) / 256) * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static __device__ __align__(256) dn::PruneView g_noalloc_views[kNoAllocMaxViews];

// The view table travels as a kernel argument (17 x 224 bytes, inside the
// 4 KB parameter space) and one block writes it into g_noalloc_views, in
// stream order: no host buffer has to outlive the call, and no copy from
// pageable host memory waits for the stream's earlier work.
struct NoAllocTable {
  dn::PruneView v[kNoAllocMaxViews];
};
static_assert(sizeof(NoAllocTable) + 16 <= 4096, "view table must fit the kernel parameters");

__global__ void install_views_kernel(NoAllocTable table, int n) {
  const int k = threadIdx.x;
  if (k < n) g_noalloc_views[k] = table.v[k];
}

bool finite_all(const double* a, int n) {
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(a[i])) return false;
  return true;
}

// The checks dn_pruner_add_view makes: finite K, R, t and an invertible K.
bool camera_ok(const dn_prune_view& v) {
  if (!finite_all(v.K, 9) || !finite_all(v.R, 9) || !finite_all(v.t, 3)) return false;
  const double* a = v.K;
  const double det = a[0] * (a[4] * a[8] - a[7] * a[5]) - a[1] * (a[3] * a[8] - a[6] * a[5]) +
                     a[2] * (a[3] * a[7] - a[6] * a[4]);
  return det != 0.0 && std::isfinite(det);
}

constexpr int kMaxDevices = 64;
struct DeviceAddrs {
  void* scratch = nullptr;
  dn::PruneView* views = nullptr;
};
DeviceAddrs g_addrs[kMaxDevices];
std::mutex g_addrs_mu;

thread_local std::string g_noalloc_error;

dn_status fail(dn_status s, const std::string& m) {
  g_noalloc_error = m;
  return s;
}

}  // namespace

extern "C" const char* dn_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

extern "C" dn_status dn_prune_noalloc(const dn_prune_view* views, int n_views,
                                      float same_depth_threshold, float* points, float* normals,
                                      uint8_t* colors, uint8_t* labels, int64_t capacity,
                                      unsigned long long* count, void* stream) {
  if (!views || !points || !normals || !colors || !labels || !count)
    return fail(DN_INVALID_ARG, "NULL argument");
  if (n_views < 1 || n_views > kNoAllocMaxViews)
    return fail(DN_INVALID_ARG, "n_views must be 1..17");
  const int W = views[0].width, H = views[0].height;
  if (W < 1 || H < 1) return fail(DN_INVALID_ARG, "bad reference depthmap size");
  if ((long long)W * H > kNoAllocMaxPixels)
    return fail(DN_INVALID_ARG,
                "reference depthmap exceeds the 4194304-pixel maximum of the static scratch");
  if (dn::prune_scratch_bytes(W, H) > kNoAllocScratchBytes)
    return fail(DN_INVALID_ARG, "static scratch too small for this depthmap");
  if (capacity < (int64_t)W * H)
    return fail(DN_INVALID_ARG, "output capacity must be at least width * height points");
  for (int k = 0; k < n_views; ++k) {
    const dn_prune_view& v = views[k];
    if (!v.depth || !v.plane || !v.color || !v.label || v.width < 1 || v.height < 1 ||
        v.width > 16384 || v.height > 16384)
      return fail(DN_INVALID_ARG, "view with NULL buffer or a size outside 1..16384");
    if (!camera_ok(v)) return fail(DN_INVALID_ARG, "camera K, R, t must be finite, K invertible");
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(DN_DEVICE_ERROR, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(DN_DEVICE_ERROR, "device index out of range");
  DeviceAddrs addrs;
  {
    std::lock_guard<std::mutex> lock(g_addrs_mu);
    if (!g_addrs[dev].scratch) {
      void* s = nullptr;
      void* v = nullptr;
      e = cudaGetSymbolAddress(&s, g_noalloc_scratch);
      if (e != cudaSuccess) return fail(DN_DEVICE_ERROR, cudaGetErrorString(e));
      e = cudaGetSymbolAddress(&v, g_noalloc_views);
      if (e != cudaSuccess) return fail(DN_DEVICE_ERROR, cudaGetErrorString(e));
      g_addrs[dev].scratch = s;
      g_addrs[dev].views = static_cast<dn::PruneView*>(v);
    }
    addrs = g_addrs[dev];
  }
  NoAllocTable table{};
  for (int k = 0; k < n_views; ++k) {
    const dn_prune_view& v = views[k];
    dn::PruneView p{};
    p.depth = v.depth;
    p.plane = v.plane;
    p.color = v.color;
    p.label = v.label;
    p.W = v.width;
    p.H = v.height;
    p.plane_stride = 3;
    for (int i = 0; i < 9; ++i) {
      p.K[i] = v.K[i];
      p.R[i] = v.R[i];
    }
    for (int i = 0; i < 3; ++i) p.t[i] = v.t[i];
    table.v[k] = p;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  install_views_kernel<<<1, 32, 0, s>>>(table, n_views);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(DN_DEVICE_ERROR, cudaGetErrorString(e));
  dn::PruneOut out{points, normals, colors, labels};
  e = dn::launch_prune(addrs.views, n_views, W, H, same_depth_threshold, addrs.scratch, out, count,
                       s);
  if (e != cudaSuccess) return fail(DN_DEVICE_ERROR, cudaGetErrorString(e));
  return DN_OK;
}
