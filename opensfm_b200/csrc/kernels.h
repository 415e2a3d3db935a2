// Host-side entry points of the dense kernels (kernels.cu, cleanprune.cu).
#pragma once

#include <algorithm>

#include "common.cuh"

namespace dn {

enum class Stage { kInit, kBruteForce, kScorePlanes, kHalfPass, kPostProcess };

struct LaunchArgs {
  const MapDev* maps;
  const ViewDev* views;
  const PairDev* pairs;
  const int4* tiles;  // (map, tile_x, tile_y, 0) per block
  int n_tiles;
  int bx, by;         // block shape (threads)
  int flag;           // post-process: apply the median filter
  RunParams p;
};

cudaError_t launch_stage(Stage stage, bool sample, const LaunchArgs& a, cudaStream_t s);
// An active-pixel half-pass in list mode (a.tiles: the half-pass tiles;
// p.active, p.pass >= 2): lists the active pixels of the colour into
// MapDev::alist in tile order (their number into MapDev::acount), chunk
// offsets into chunk0 (n_maps + 1 ints), then the half-pass over the lists.
// tile_count and tile_off: scratch of a.n_tiles ints each.
cudaError_t launch_halfpass_list(bool sample, const LaunchArgs& a, int n_maps, int* chunk0,
                                 int* tile_count, int* tile_off, cudaStream_t s);

struct CleanView;
struct CleanMap;
struct PruneMap;
// The cleaner and pruner stages of the persistent launch (n_clean == 0:
// none; n_prune == 0: no pruner).  Tiles as launch_clean_batch and
// launch_prune_batch take them.
struct PersistentTail {
  const CleanView* clean_views;
  const CleanMap* cmaps;
  const int* lists;
  const int4* clean_tiles;
  int n_clean;
  int min_views;
  float thr;
  int n_pmaps;
  const PruneMap* pmaps;
  const int4* prune_tiles;
  int n_prune;
  int pad_;
};
// A whole PatchMatch run (7 x 7 patch, non-sample) in one cooperative
// persistent launch: init tiles, n_half half-pass stages, post tiles, then
// the cleaner and the pruner's three stages over every map.
struct PersistentArgs {
  LaunchArgs base;
  const int4* tiles_init;
  int n_init;
  const int4* tiles_hp;
  int n_hp;
  const int4* tiles_post;
  int n_post;
  int n_half;
  unsigned* sync;  // kPersistentCounters + n_half counters, zeroed before the launch
  PersistentTail tail;
};
// Barrier words and stage counters of the persistent launch besides the
// n_half half-pass counters: arrivals, generation, init, post, clean,
// prune flags, scan, prune writes.
constexpr int kPersistentCounters = 8;
cudaError_t launch_persistent(const PersistentArgs& pa, cudaStream_t s);
// The persistent launch's grid barrier with a barrier that never opens
// (`blocks` blocks, one more expected): returns with *error = 1 after at
// most max_spins polls of 100 ns per block.  sync: 2 zeroed words.
cudaError_t launch_barrier_expiry(unsigned* sync, int* error, int blocks, long long max_spins,
                                  cudaStream_t s);
cudaError_t launch_prepare_view(const uint8_t* d_u8, int W, int H, int stride, __half* d_img,
                                uint2* d_quad, int TP, int TW, int TH, float cbias,
                                cudaStream_t s);

// Re-uploaded views prepared together: per job, the u8 pixels at `src`
// (W x H, packed) become the view's u8 copy, FP16 image and coefficient
// table (the same values as launch_prepare_view) in one pass.  Any n; one
// launch per kPrepareJobs jobs (the jobs travel as kernel parameters).
struct PrepareJob {
  const uint8_t* src;
  uint8_t* gray;
  __half* img;
  uint2* quad;
  int W, H, TP, TW, TH;
  float cbias;
};
constexpr int kPrepareJobs = 48;
cudaError_t launch_prepare_views(const PrepareJob* jobs, int n, cudaStream_t s);

// Packs n float arrays (src[k], count[k] floats) into dst, array k at
// dst + off[k]; every off[k] a multiple of 4.  One launch per kGatherArrays.
constexpr int kGatherArrays = 96;
cudaError_t launch_gather_floats(const float* const* src, const size_t* count, const size_t* off,
                                 int n, float* dst, cudaStream_t s);

// Table geometry of a W x H view: used width TW = W - 1 + 2P, rows
// TH = H - 1 + 2P, pitch TP = 1024 k - 1 >= TW (k a power of two) and the
// floor constant M = 2^23 + 2^22 / k (see ViewDev).
struct TableGeom {
  int TW, TH, TP;
  float magic;
};
inline TableGeom table_geom(int W, int H) {
  TableGeom g;
  g.TW = W - 1 + 2 * kPad;
  g.TH = H - 1 + 2 * kPad;
  int k = 1;
  while (1024 * k - 1 < g.TW) k *= 2;
  g.TP = 1024 * k - 1;
  g.magic = 8388608.0f + 4194304.0f / (float)k;
  return g;
}
cudaError_t launch_pack(const MapDev* maps, int map, float* plane, size_t n, cudaStream_t s);
cudaError_t launch_postprocess_plain(const float* in, float* out, int W, int H, cudaStream_t s);
cudaError_t fp32_peak(double* tflops, double* ms);
// G taps/s of walk_ceiling_kernel (the table walk and its sums alone) on a
// 1024 x 768 view, 64 walks per pixel.
cudaError_t walk_ceiling(double* gtaps, double* ms);

// Cleaner / pruner (cleanprune.cu).
struct CleanView {
  const float* depth;  // [H][W]
  int W, H, stride;
  double K[9], R[9], t[3];
};
struct PruneView {
  const float* depth;    // [H][W]
  const float* plane;    // [H][W][plane_stride], plane v in the first 3 floats
  const uint8_t* color;  // [H][W][3], or null: gray replicated to 3 channels
  const uint8_t* label;  // [H][W], or null: label 0
  int W, H;
  double K[9], R[9], t[3];
  const uint8_t* gray;   // [H][W] used when color is null
  int plane_stride;      // floats per pixel in `plane` (3, or 4 for PatchMatch state)
  int pad_;
};
struct PruneOut {
  float* points;
  float* normals;
  uint8_t* colors;
  uint8_t* labels;
};

// Cleans map `ref` against views others[0..n) (DepthmapCleaner::Clean).
cudaError_t launch_clean(const CleanView* d_views, int ref, const int* d_others, int n_others,
                         int W, int H, float thr, int min_views, float* out, cudaStream_t s);
// Every map of a batch in one launch: map k (CleanView k, reference of the
// k-th map) against the views lists[cmaps[k].list_off ..][0..cmaps[k].n),
// into cmaps[k].out; tiles (map, tx, ty) of kCleanTileX x kCleanTileY px.
constexpr int kCleanTileX = 32, kCleanTileY = 4;
struct CleanMap {
  int list_off, n, pad_[2];
  float* out;  // [H][W] cleaned depth
};
cudaError_t launch_clean_batch(const CleanView* d_views, const CleanMap* d_cmaps,
                               const int* d_lists, const int4* d_tiles, int n_tiles, float thr,
                               int min_views, cudaStream_t s);
// GPUDepthmapCleaner::Clean (cleaner.cc:56-170): forward and backward
// consistency with space carving, FP32, every source the reference's size.
constexpr int kMaxGpuCleanSources = 16;
struct GpuCleanCam {
  float K[9], R[9], t[3];
};
struct GpuCleanArgs {
  const float* ref;                           // [H][W]
  const float* src[kMaxGpuCleanSources];      // [H][W] each
  GpuCleanCam cam[kMaxGpuCleanSources + 1];   // reference first
  int W, H, n_src;
  float same_depth_threshold;
  int min_consistent;
  float carving_threshold;
  int max_carved;
};
cudaError_t launch_gpu_clean(const GpuCleanArgs& a, float* out, cudaStream_t s);
// Pruner in three kernels: keep flags + per-block counts, block-count scan,
// ordered compaction.  `scratch` holds ceil(W*H/1024) + 1 uint32 counts and
// W*H keep bytes (see prune_scratch_bytes).
size_t prune_scratch_bytes(int W, int H);
cudaError_t launch_prune(const PruneView* d_views, int n_views, int W, int H, float thr,
                         void* scratch, PruneOut out, unsigned long long* d_count, cudaStream_t s);
// The pruner over every map of a batch: flags over tiles (map, block) of
// kPruneBatchBlock pixels, one scan block per map, ordered writes; three
// launches in all.  Same output order as launch_prune (row-major).
constexpr int kPruneBatchBlock = 128;
struct PruneMap {
  const PruneView* views;  // this map first
  int n_views, blocks;     // blocks of kPruneBatchBlock pixels
  uint8_t* keep;           // [H][W]
  uint32_t* counts;        // [blocks]
  uint32_t* offsets;       // [blocks + 1]
  PruneOut out;
  unsigned long long* count;
};
size_t prune_batch_scratch_bytes(int W, int H);
PruneMap prune_batch_map(const PruneView* d_views, int n_views, int W, int H, void* scratch,
                         PruneOut out, unsigned long long* d_count);
cudaError_t launch_prune_batch(const PruneMap* d_pm, int n_maps, const int4* d_tiles, int n_tiles,
                               float thr, cudaStream_t s);

}  // namespace dn
