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
    if (!v.depth || !v.plane || !v.color || !v.label || v.width < 1 || v.height < 1)
      return fail(DN_INVALID_ARG, "view with NULL buffer or bad size");
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
  dn::PruneView table[kNoAllocMaxViews];
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
    table[k] = p;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  e = cudaMemcpyAsync(addrs.views, table, n_views * sizeof(dn::PruneView), cudaMemcpyHostToDevice,
                      s);
  if (e != cudaSuccess) return fail(DN_DEVICE_ERROR, cudaGetErrorString(e));
  dn::PruneOut out{points, normals, colors, labels};
  e = dn::launch_prune(addrs.views, n_views, W, H, same_depth_threshold, addrs.scratch, out, count,
                       s);
  if (e != cudaSuccess) return fail(DN_DEVICE_ERROR, cudaGetErrorString(e));
  return DN_OK;
}
