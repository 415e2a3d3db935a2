// Host engine and C ABI (include/dense_b200.h) of the dense depthmap library.
//
// One Engine holds a reconstruction's views (uploaded once, FP16 image +
// bilinear coefficient table per view) and its depthmaps (reference view,
// matching views, depth range, per-map state).  The legacy single-depthmap
// classes (DepthmapEstimator / Cleaner / Pruner, reference
// opensfm/src/lib/dense/depthmap.h:57-153) are thin wrappers over it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "dense_b200.h"
#include "device_guard.h"
#include "kernels.h"
#include "learned.h"

namespace {

thread_local std::string g_last_error;

dn_status fail(dn_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

dn_status cuda_fail(cudaError_t e, const char* what) {
  const dn_status s = (e == cudaErrorMemoryAllocation) ? DN_OUT_OF_MEMORY : DN_DEVICE_ERROR;
  return fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

#define DN_CUDA(expr)                                        \
  do {                                                       \
    cudaError_t e_ = (expr);                                 \
    if (e_ != cudaSuccess) return cuda_fail(e_, #expr);      \
  } while (0)

#define DN_CHECK(cond, msg)                                  \
  do {                                                       \
    if (!(cond)) return fail(DN_INVALID_ARG, msg);           \
  } while (0)

#define DN_TRY(expr)                                         \
  do {                                                       \
    dn_status s_ = (expr);                                   \
    if (s_ != DN_OK) return s_;                              \
  } while (0)

// Device buffer owned by the host object.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  cudaError_t alloc(size_t count) {
    if (count <= n && p) return cudaSuccess;
    release();
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
    if (e == cudaSuccess) n = count;
    else p = nullptr;
    return e;
  }
};

// ---------------------------------------------------------------- FP64 math
// 3x3 helpers in the evaluation order of cv::Matx (products accumulate from
// zero in index order); the inverse is the cofactor form scaled by 1/det.
void m3_mul(const double* a, const double* b, double* c) {
  double r[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += a[3 * i + k] * b[3 * k + j];
      r[3 * i + j] = s;
    }
  std::memcpy(c, r, sizeof(r));
}
void m3_vec(const double* a, const double* x, double* y) {
  double r[3];
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s += a[3 * i + k] * x[k];
    r[i] = s;
  }
  std::memcpy(y, r, sizeof(r));
}
void m3_t(const double* a, double* b) {
  double r[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[3 * j + i] = a[3 * i + j];
  std::memcpy(b, r, sizeof(r));
}
bool m3_inv(const double* a, double* r) {
  auto A = [&](int i, int j) { return a[3 * i + j]; };
  double d = A(0, 0) * (A(1, 1) * A(2, 2) - A(2, 1) * A(1, 2)) -
             A(0, 1) * (A(1, 0) * A(2, 2) - A(2, 0) * A(1, 2)) +
             A(0, 2) * (A(1, 0) * A(2, 1) - A(2, 0) * A(1, 1));
  if (d == 0 || !std::isfinite(d)) return false;
  d = 1 / d;
  r[0] = (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) * d;
  r[1] = (A(0, 2) * A(2, 1) - A(0, 1) * A(2, 2)) * d;
  r[2] = (A(0, 1) * A(1, 2) - A(0, 2) * A(1, 1)) * d;
  r[3] = (A(1, 2) * A(2, 0) - A(1, 0) * A(2, 2)) * d;
  r[4] = (A(0, 0) * A(2, 2) - A(0, 2) * A(2, 0)) * d;
  r[5] = (A(0, 2) * A(1, 0) - A(0, 0) * A(1, 2)) * d;
  r[6] = (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0)) * d;
  r[7] = (A(0, 1) * A(2, 0) - A(0, 0) * A(2, 1)) * d;
  r[8] = (A(0, 0) * A(1, 1) - A(0, 1) * A(1, 0)) * d;
  return true;
}
bool all_finite(const double* a, int n) {
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(a[i])) return false;
  return true;
}

struct Camera {
  double K[9], R[9], t[3];
};

dn_status check_camera(const double* K, const double* R, const double* t) {
  DN_CHECK(K && R && t, "K, R and t must not be NULL");
  DN_CHECK(all_finite(K, 9) && all_finite(R, 9) && all_finite(t, 3),
           "camera K, R, t must be finite");
  double Ki[9];
  DN_CHECK(m3_inv(K, Ki), "camera K is singular");
  return DN_OK;
}

// ---------------------------------------------------------------- engine
struct View {
  Camera cam;
  int W = 0, H = 0;
  float cbias = 0.f;
  DevBuf<__half> img;
  DevBuf<uint8_t> mask;
  DevBuf<uint2> quad;  // bilinear coefficient table, 4 x FP16 per entry
  DevBuf<uint8_t> gray;  // u8 copy (pruner colour when none is given)
  // Pipelined replacement of the pixels (dn_batch_upload_view_image): the
  // host copy lands here on the upload stream.
  DevBuf<uint8_t> upload;
};

struct Map {
  int ref = 0;
  std::vector<int> nbrs;  // view ids
  double min_d = 0, max_d = 0;
  std::vector<int> clean_maps;
  DevBuf<float4> state;
  DevBuf<float> score, depth, clean, init, plane_out;
  DevBuf<int> nghbr;
  bool has_init = false;
  DevBuf<float> prop_init;   // learned proposal planes [H][W][3]
  DevBuf<uint8_t> changed;   // active-pixel flags [H][W]
  DevBuf<int> alist;         // active-pixel list of a half-pass [H W]
  // Pruner (DN_RUN_PRUNE): views (this map first), scratch, outputs.
  DevBuf<dn::PruneView> prune_views;
  DevBuf<uint8_t> prune_scratch, prune_colors, prune_labels;
  DevBuf<float> prune_points, prune_normals;
};

enum class Mode { kBruteForce, kPatchMatch, kPatchMatchSample, kScorePlanes };

struct Engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<std::unique_ptr<View>> views;
  std::vector<std::unique_ptr<Map>> maps;
  int patch = 7;
  float min_var = 25.f;
  int iterations = 3;
  int num_planes = 50;
  uint64_t seed = 0x5EEDBA5Eull;
  float same_depth_thr = 0.01f;
  int min_consistent = 2;
  int bx = 32, by = 4;  // thread block shape
  int variant = 2;      // lanes per pixel in init / half-passes (1, 2, 4, 8); 2 measured fastest
  int half_passes = -1;  // -1: 2 x iterations
  int persistent = 0;    // one cooperative persistent launch per PatchMatch run
  DevBuf<unsigned> d_sync;
  int use_near = 1, use_far = 1, n_refine = 6;
  float depth_range0 = 0.02f, normal_range0 = 0.5f;
  int sample_hp = 0;  // half-passes score one view per candidate (sample mode)
  int use_knight = 0;  // knight-move candidates in the half-passes
  int active = 0;     // active-pixel half-passes
  float active_tol = 0.f;
  int active_lists = 1;  // active half-passes on compacted pixel lists
  float seed_score = 0.f;  // > 0: settled start below this initial score (see RunParams)
  int init_fallback = 0;   // given / learned planes: random plane where it scores higher
  DevBuf<int> d_acount, d_chunk0;  // per map: listed pixels; chunk offsets
  DevBuf<int> d_tile_count, d_tile_off;  // per half-pass tile: active pixels, list offset
  // Learned proposal (DN_RUN_LEARNED): network weights, the feature grid of
  // every map (maps of one grid size contiguous, one network launch per
  // size), activations and outputs.
  struct PropGroup {
    int W, H, n;
    long long off;  // first grid point
    int S;          // grid stride of its maps
  };
  bool prop_on = false;
  int prop_stride = 2, prop_planes = 8;
  int prop_ref_dim = 0;  // larger side of the training images (0: one stride for every map)
  struct SweepRange {
    int S, first, count;  // sweep tiles of the maps of grid stride S
  };
  std::vector<SweepRange> sweep_ranges;
  // The proposal-grid stride of a map: the network's stride scaled by the
  // map's larger side over the training images' (prop_ref_dim > 0), rounded
  // down to 1, 2, 4 or 8, so that every map's grid has the scale the network
  // was trained at; with prop_ref_dim = 0 the network's stride.
  int map_prop_stride(const View& r) const {
    if (prop_ref_dim <= 0) return prop_stride;
    const double s = (double)prop_stride * std::max(r.W, r.H) / prop_ref_dim;
    int k = 1;
    while (k < 8 && 2.0 * k <= s) k *= 2;
    return k;
  }
  DevBuf<__nv_bfloat16> d_prop_w;
  DevBuf<float> d_prop_b;
  DevBuf<__nv_bfloat16> d_feat, d_act0, d_act1;
  DevBuf<float> d_prop_out;
  DevBuf<int4> d_tiles_prop, d_tiles_sweep;
  int n_tiles_prop = 0, prop_max_pixels = 0;
  std::vector<PropGroup> prop_groups;
  DevBuf<dn::ViewDev> d_views;
  DevBuf<dn::PairDev> d_pairs;
  DevBuf<dn::MapDev> d_maps;
  DevBuf<int4> d_tiles1, d_tiles2, d_tiles_init;
  int n_tiles1 = 0, n_tiles2 = 0, n_tiles_init = 0;
  DevBuf<unsigned long long> d_taps;
  DevBuf<int> d_error;
  DevBuf<dn::CleanView> d_clean_views;
  DevBuf<int> d_clean_lists;
  bool dirty = true;
  bool computed = false;
  cudaGraphExec_t graph = nullptr;
  unsigned graph_flags = 0;
  Mode graph_mode = Mode::kPatchMatch;
  // run start, init, half-passes, post, clean, timer x2, proposal
  static constexpr int kEvents = 8;
  bool timed_learned = false;
  cudaEvent_t ev[kEvents] = {};
  bool timed = false;
  // Pipelined host I/O: uploads run on `up` and readbacks on `down`, beside
  // the work on the batch stream (two streams, so that the next step's
  // uploads do not queue behind a readback that waits for the current run).
  // - An upload copies the pixels into the view's upload buffer on `up` and
  //   lists the view as pending.  The next work on the batch stream that
  //   reads views (flush_uploads) waits for `up` (ev_uploaded), prepares
  //   every pending view in one launch, and records ev_consumed, which later
  //   uploads wait for before they overwrite an upload buffer.
  // - A readback gathers the depths into one of two device staging buffers
  //   on the batch stream (ev_staged), then copies them to the host on
  //   `down` (ev_stage_done[k]: staging buffer k is free again).
  cudaStream_t up = nullptr, down = nullptr;
  std::vector<int> pending_uploads;
  DevBuf<float> d_stage[2];
  cudaEvent_t ev_uploaded = nullptr, ev_consumed = nullptr;
  cudaEvent_t ev_staged = nullptr, ev_stage_done[2] = {}, ev_io_tail[2] = {};
  int stage_next = 0;

  ~Engine() {
    if (graph) cudaGraphExecDestroy(graph);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : {ev_uploaded, ev_consumed, ev_staged, ev_stage_done[0],
                          ev_stage_done[1], ev_io_tail[0], ev_io_tail[1]})
      if (e) cudaEventDestroy(e);
    if (up) cudaStreamDestroy(up);
    if (down) cudaStreamDestroy(down);
    if (stream) cudaStreamDestroy(stream);
  }

  dn_status init() {
    DN_CUDA(cudaGetDevice(&device));
    DN_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    DN_CUDA(cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking));
    DN_CUDA(cudaStreamCreateWithFlags(&down, cudaStreamNonBlocking));
    DN_CUDA(d_taps.alloc(4));
    DN_CUDA(d_error.alloc(1));
    for (auto& e : ev) DN_CUDA(cudaEventCreate(&e));
    for (cudaEvent_t* e : {&ev_uploaded, &ev_consumed, &ev_staged, &ev_stage_done[0],
                           &ev_stage_done[1], &ev_io_tail[0], &ev_io_tail[1]})
      DN_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return DN_OK;
  }

  // Prepares the views uploaded since the last flush, in stream order on the
  // batch stream (see `up` above).
  dn_status flush_uploads() {
    if (pending_uploads.empty()) return DN_OK;
    DN_CUDA(cudaSetDevice(device));
    DN_CUDA(cudaEventRecord(ev_uploaded, up));
    DN_CUDA(cudaStreamWaitEvent(stream, ev_uploaded, 0));
    std::vector<dn::PrepareJob> jobs;
    jobs.reserve(pending_uploads.size());
    for (int v : pending_uploads) {
      View& w = *views[v];
      const dn::TableGeom tg = dn::table_geom(w.W, w.H);
      jobs.push_back({w.upload.p, w.gray.p, w.img.p, w.quad.p, w.W, w.H, tg.TP, tg.TW, tg.TH,
                      w.cbias});
    }
    pending_uploads.clear();
    DN_CUDA(dn::launch_prepare_views(jobs.data(), (int)jobs.size(), stream));
    DN_CUDA(cudaEventRecord(ev_consumed, stream));
    return DN_OK;
  }

  // Makes the batch stream wait for everything enqueued on the I/O streams.
  dn_status join_io() {
    DN_CUDA(cudaEventRecord(ev_io_tail[0], up));
    DN_CUDA(cudaEventRecord(ev_io_tail[1], down));
    DN_CUDA(cudaStreamWaitEvent(stream, ev_io_tail[0], 0));
    DN_CUDA(cudaStreamWaitEvent(stream, ev_io_tail[1], 0));
    return DN_OK;
  }

  dn_status mark(int k, bool on) {
    if (on) DN_CUDA(cudaEventRecord(ev[k], stream));
    return DN_OK;
  }

  void invalidate() {
    dirty = true;
    computed = false;
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
  }

  dn_status add_view(const double* K, const double* R, const double* t, const uint8_t* image,
                     const uint8_t* mask, int W, int H, int stride, int* id) {
    DN_TRY(check_camera(K, R, t));
    DN_CHECK(image, "image must not be NULL");
    DN_CHECK(W >= 2 && H >= 2 && W <= 16384 && H <= 16384, "image size must be 2..16384");
    if (stride <= 0) stride = W;
    DN_CHECK(stride >= W, "stride must be >= width");
    DN_CUDA(cudaSetDevice(device));
    auto v = std::make_unique<View>();
    std::memcpy(v->cam.K, K, sizeof(v->cam.K));
    std::memcpy(v->cam.R, R, sizeof(v->cam.R));
    std::memcpy(v->cam.t, t, sizeof(v->cam.t));
    v->W = W;
    v->H = H;
    // Centring constant: the rounded mean intensity (an integer, so the
    // coefficient table stays exact).
    double sum = 0;
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x) sum += image[(size_t)y * stride + x];
    v->cbias = (float)std::floor(sum / ((double)W * H) + 0.5);
    const dn::TableGeom tg = dn::table_geom(W, H);
    DN_CHECK(W <= 8192 - 2 * dn::kPad, "image wider than the table layout supports (8176)");
    DN_CUDA(v->img.alloc((size_t)W * H));
    DN_CUDA(v->quad.alloc((size_t)tg.TP * tg.TH));
    DN_CUDA(v->gray.alloc((size_t)W * H));
    DN_CUDA(cudaMemcpy2DAsync(v->gray.p, W, image, stride, W, H, cudaMemcpyHostToDevice, stream));
    if (mask) {
      DN_CUDA(v->mask.alloc((size_t)W * H));
      DN_CUDA(cudaMemcpy2DAsync(v->mask.p, W, mask, stride, W, H, cudaMemcpyHostToDevice, stream));
    }
    DN_CUDA(dn::launch_prepare_view(v->gray.p, W, H, W, v->img.p, v->quad.p, tg.TP, tg.TW, tg.TH,
                                    v->cbias, stream));
    DN_CUDA(cudaStreamSynchronize(stream));
    if (id) *id = (int)views.size();
    views.push_back(std::move(v));
    invalidate();
    return DN_OK;
  }

  dn_status add_map(int ref, const int* nbrs, int n, double min_d, double max_d, int* id) {
    DN_CHECK(ref >= 0 && ref < (int)views.size(), "reference view id out of range");
    DN_CHECK(n >= 1 && n <= dn::kMaxNbr, "a depthmap needs 1..16 matching views");
    auto m = std::make_unique<Map>();
    m->ref = ref;
    for (int k = 0; k < n; ++k) {
      DN_CHECK(nbrs[k] >= 0 && nbrs[k] < (int)views.size(), "matching view id out of range");
      m->nbrs.push_back(nbrs[k]);
    }
    m->min_d = min_d;
    m->max_d = max_d;
    if (id) *id = (int)maps.size();
    maps.push_back(std::move(m));
    invalidate();
    return DN_OK;
  }

  dn_status check_params(Mode mode) {
    DN_CHECK(!maps.empty(), "no depthmap declared (add at least two views)");
    const int hpz = (patch - 1) / 2;
    DN_CHECK(hpz >= 1 && hpz <= dn::kMaxHpz, "patch size must be in 3..12");
    for (auto& m : maps) {
      const View& r = *views[m->ref];
      DN_CHECK(r.W > 2 * hpz && r.H > 2 * hpz, "image smaller than the patch");
      if (mode == Mode::kBruteForce) {
        DN_CHECK(num_planes >= 2, "brute force needs at least 2 depth planes");
        DN_CHECK(m->min_d > 0 && m->max_d > 0 && std::isfinite(m->min_d) && std::isfinite(m->max_d),
                 "depth range must be positive and finite");
      }
      if (mode == Mode::kPatchMatch || mode == Mode::kPatchMatchSample) {
        DN_CHECK(m->min_d > 0 && m->max_d > 0 && std::isfinite(m->min_d) && std::isfinite(m->max_d),
                 "depth range must be positive and finite");
        DN_CHECK(iterations >= 0 && iterations <= 1000, "iterations must be 0..1000");
      }
    }
    return DN_OK;
  }

  // Builds the per-pair homography factors (FP64) and the device tables.
  dn_status prepare() {
    DN_TRY(flush_uploads());
    if (!dirty) return DN_OK;
    DN_CUDA(cudaSetDevice(device));
    std::vector<dn::ViewDev> hv(views.size());
    for (size_t k = 0; k < views.size(); ++k) {
      const View& v = *views[k];
      dn::ViewDev d{};
      const dn::TableGeom tg = dn::table_geom(v.W, v.H);
      d.img = v.img.p;
      d.mask = v.mask.p;
      d.quad = v.quad.p;
      d.quad0 = v.quad.p + (size_t)dn::kPad * tg.TP + dn::kPad;
      d.W = v.W;
      d.H = v.H;
      d.TP = tg.TP;
      d.TH = tg.TH;
      d.cbias = v.cbias;
      d.magic = tg.magic;
      hv[k] = d;
    }
    std::vector<dn::PairDev> hp;
    std::vector<dn::MapDev> hm(maps.size());
    std::vector<int4> t1, t2, ti, tp;
    const int lanes = (patch == 7) ? variant : 1;
    // Proposal grid: every map at its own stride; maps grouped by grid size
    // and stride in order of first appearance, each group's maps contiguous.
    std::vector<long long> prop_off(maps.size(), 0);
    std::vector<int> prop_s(maps.size(), prop_stride);
    prop_groups.clear();
    prop_max_pixels = 0;
    long long prop_points = 0;
    if (prop_on) {
      for (size_t a = 0; a < maps.size(); ++a) prop_s[a] = map_prop_stride(*views[maps[a]->ref]);
      std::vector<int> done(maps.size(), 0);
      for (size_t a = 0; a < maps.size(); ++a) {
        if (done[a]) continue;
        const View& ra = *views[maps[a]->ref];
        const int S = prop_s[a];
        PropGroup g{(ra.W + S - 1) / S, (ra.H + S - 1) / S, 0, prop_points, S};
        for (size_t b2 = a; b2 < maps.size(); ++b2) {
          const View& rb = *views[maps[b2]->ref];
          if (done[b2] || prop_s[b2] != S || (rb.W + S - 1) / S != g.W ||
              (rb.H + S - 1) / S != g.H)
            continue;
          done[b2] = 1;
          prop_off[b2] = prop_points;
          prop_points += (long long)g.W * g.H;
          ++g.n;
        }
        prop_groups.push_back(g);
      }
    }
    std::vector<std::vector<int4>> tp_by_s(4);  // sweep tiles of strides 1, 2, 4, 8
    if (active) {
      DN_CUDA(d_acount.alloc(maps.size()));
      DN_CUDA(d_chunk0.alloc(maps.size() + 1));
    }
    for (size_t mi = 0; mi < maps.size(); ++mi) {
      Map& m = *maps[mi];
      const View& r = *views[m.ref];
      const size_t npx = (size_t)r.W * r.H;
      DN_CUDA(m.state.alloc(npx));
      DN_CUDA(m.score.alloc(npx));
      DN_CUDA(m.depth.alloc(npx));
      DN_CUDA(m.nghbr.alloc(npx));
      double Kinv[9], R0t[9];
      m3_inv(r.cam.K, Kinv);
      m3_t(r.cam.R, R0t);
      dn::MapDev d{};
      d.ref_view = m.ref;
      d.W = r.W;
      d.H = r.H;
      d.n_pairs = (int)m.nbrs.size();
      d.pair0 = (int)hp.size();
      for (int k = 0; k < 9; ++k) {
        d.Kinv[k] = (float)Kinv[k];
        d.Kinv_d[k] = Kinv[k];
        d.K[k] = r.cam.K[k];
        d.R[k] = r.cam.R[k];
      }
      for (int k = 0; k < 3; ++k) d.t[k] = r.cam.t[k];
      d.log_min = (float)std::log(m.min_d);
      d.log_max = (float)std::log(m.max_d);
      d.min_depth = m.min_d;
      d.max_depth = m.max_d;
      d.state = m.state.p;
      d.score = m.score.p;
      d.nghbr = m.nghbr.p;
      d.depth = m.depth.p;
      d.clean = m.clean.p;
      d.init = m.has_init ? m.init.p : nullptr;
      if (active) {
        DN_CUDA(m.changed.alloc(npx));
        d.changed = m.changed.p;
        DN_CUDA(m.alist.alloc(npx));
        d.alist = m.alist.p;
        d.acount = d_acount.p + mi;
      }
      if (prop_on) {
        DN_CUDA(m.prop_init.alloc(3 * npx));
        d.prop_init = m.prop_init.p;
        d.prop_off = prop_off[mi];
        d.prop_S = prop_s[mi];
        d.prop_W = (r.W + d.prop_S - 1) / d.prop_S;
        d.prop_H = (r.H + d.prop_S - 1) / d.prop_S;
        prop_max_pixels = std::max(prop_max_pixels, r.W * r.H);
        // Sweep tiles: (bx / lanes) x by grid points per block, one list per
        // stride (the sweep kernel is compiled per stride).
        const int pxs = bx / lanes;
        const int si = d.prop_S == 1 ? 0 : (d.prop_S == 2 ? 1 : (d.prop_S == 4 ? 2 : 3));
        for (int y = 0; y < (d.prop_H + by - 1) / by; ++y)
          for (int x = 0; x < (d.prop_W + pxs - 1) / pxs; ++x)
            tp_by_s[si].push_back(make_int4((int)mi, x, y, 0));
      }
      for (int o : m.nbrs) {
        const View& ov = *views[o];
        // Q = R_o R_0^T, a = Q t_0 - t_o (depthmap.cc:152-155);
        // H(v) = K_o (Q + a v^T) K_0^-1 = G + e f^T, G = K_o Q K_0^-1,
        // e = K_o a, f = K_0^-T v.
        double Q[9], qt[3], a[3], G[9], T[9], e[3];
        m3_mul(ov.cam.R, R0t, Q);
        m3_vec(Q, r.cam.t, qt);
        for (int k = 0; k < 3; ++k) a[k] = qt[k] - ov.cam.t[k];
        m3_mul(ov.cam.K, Q, T);
        m3_mul(T, Kinv, G);
        m3_vec(ov.cam.K, a, e);
        dn::PairDev p{};
        for (int k = 0; k < 9; ++k) p.G[k] = (float)G[k];
        for (int k = 0; k < 3; ++k) p.e[k] = (float)e[k];
        p.view = o;
        hp.push_back(p);
      }
      hm[mi] = d;
      const int px = bx / lanes;  // pixels per warp row in init / half-passes
      const int tx1 = (r.W + bx - 1) / bx, ty1 = (r.H + by - 1) / by;
      const int tx2 = (r.W + 2 * px - 1) / (2 * px);
      const int txi = (r.W + px - 1) / px;
      hm[mi].hp_tile0 = (int)t2.size();  // the map's half-pass tiles are contiguous
      hm[mi].hp_tiles = tx2 * ty1;
      for (int y = 0; y < ty1; ++y) {
        for (int x = 0; x < tx1; ++x) t1.push_back(make_int4((int)mi, x, y, 0));
        for (int x = 0; x < tx2; ++x) t2.push_back(make_int4((int)mi, x, y, 0));
        for (int x = 0; x < txi; ++x) ti.push_back(make_int4((int)mi, x, y, 0));
      }
    }
    DN_CUDA(d_views.alloc(std::max<size_t>(hv.size(), 1)));
    DN_CUDA(d_pairs.alloc(std::max<size_t>(hp.size(), 1)));
    DN_CUDA(d_maps.alloc(std::max<size_t>(hm.size(), 1)));
    DN_CUDA(d_tiles1.alloc(std::max<size_t>(t1.size(), 1)));
    DN_CUDA(d_tiles2.alloc(std::max<size_t>(t2.size(), 1)));
    DN_CUDA(d_tiles_init.alloc(std::max<size_t>(ti.size(), 1)));
    if (active) {
      DN_CUDA(d_tile_count.alloc(std::max<size_t>(t2.size(), 1)));
      DN_CUDA(d_tile_off.alloc(std::max<size_t>(t2.size(), 1)));
    }
    DN_CUDA(cudaMemcpyAsync(d_views.p, hv.data(), hv.size() * sizeof(dn::ViewDev),
                            cudaMemcpyHostToDevice, stream));
    if (!hp.empty())
      DN_CUDA(cudaMemcpyAsync(d_pairs.p, hp.data(), hp.size() * sizeof(dn::PairDev),
                              cudaMemcpyHostToDevice, stream));
    DN_CUDA(cudaMemcpyAsync(d_maps.p, hm.data(), hm.size() * sizeof(dn::MapDev),
                            cudaMemcpyHostToDevice, stream));
    DN_CUDA(cudaMemcpyAsync(d_tiles1.p, t1.data(), t1.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, stream));
    DN_CUDA(cudaMemcpyAsync(d_tiles2.p, t2.data(), t2.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, stream));
    DN_CUDA(cudaMemcpyAsync(d_tiles_init.p, ti.data(), ti.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, stream));
    n_tiles_prop = 0;
    sweep_ranges.clear();
    if (prop_on) {
      for (int si = 0; si < 4; ++si) {
        if (tp_by_s[si].empty()) continue;
        sweep_ranges.push_back({1 << si, (int)tp.size(), (int)tp_by_s[si].size()});
        tp.insert(tp.end(), tp_by_s[si].begin(), tp_by_s[si].end());
      }
      DN_CUDA(d_tiles_prop.alloc(std::max<size_t>(tp.size(), 1)));
      DN_CUDA(cudaMemcpyAsync(d_tiles_prop.p, tp.data(), tp.size() * sizeof(int4),
                              cudaMemcpyHostToDevice, stream));
      n_tiles_prop = (int)tp.size();
      const size_t n = (size_t)std::max<long long>(prop_points, 1);
      DN_CUDA(d_feat.alloc(n * dn::kFeatC));
      DN_CUDA(d_act0.alloc(n * dn::kFeatC));
      DN_CUDA(d_act1.alloc(n * dn::kFeatC));
      DN_CUDA(d_prop_out.alloc(n * 4));
      // Grid points that no sweep thread reaches keep zero features.
      DN_CUDA(cudaMemsetAsync(d_feat.p, 0, n * dn::kFeatC * sizeof(__nv_bfloat16), stream));
    }
    DN_CUDA(cudaStreamSynchronize(stream));
    n_tiles1 = (int)t1.size();
    n_tiles2 = (int)t2.size();
    n_tiles_init = (int)ti.size();
    // Counters of the persistent launch (allocated here, outside any capture).
    const int n_half = half_passes >= 0 ? half_passes : 2 * iterations;
    DN_CUDA(d_sync.alloc(dn::kPersistentCounters + std::max(n_half, 0)));
    dirty = false;
    return DN_OK;
  }

  dn::LaunchArgs args(bool halfpass) const {
    dn::LaunchArgs a{};
    a.maps = d_maps.p;
    a.views = d_views.p;
    a.pairs = d_pairs.p;
    a.tiles = halfpass ? d_tiles2.p : d_tiles1.p;
    a.n_tiles = halfpass ? n_tiles2 : n_tiles1;
    a.bx = bx;
    a.by = by;
    a.p.hpz = (patch - 1) / 2;
    a.p.min_var = min_var;
    a.p.seed_lo = (uint32_t)seed;
    a.p.seed_hi = (uint32_t)(seed >> 32);
    a.p.num_planes = num_planes;
    a.p.same_depth_thr = same_depth_thr;
    a.p.min_consistent = min_consistent;
    a.p.taps = d_taps.p;
    a.p.error = d_error.p;
    a.p.variant = variant;
    a.p.use_near = use_near;
    a.p.use_far = use_far;
    a.p.n_refine = n_refine;
    a.p.depth_range0 = depth_range0;
    a.p.normal_range0 = normal_range0;
    a.p.active = active;
    a.p.active_tol = active_tol;
    a.p.seed_score = seed_score > 0.f ? seed_score : 3.0f;  // NCC <= 1: every pixel moved
    a.p.init_fallback = init_fallback;
    a.p.active_from = seed_score > 0.f ? 0 : 2;
    a.p.use_knight = use_knight;
    return a;
  }

  // The learned proposal of every map: feature sweep on the proposal grid,
  // the 6-layer network per grid size (tcgen05 forward), planes installed
  // into MapDev::prop_init at full resolution.
  static constexpr int kPropLayers = 6;
  dn_status enqueue_proposal() {
    DN_CHECK(prop_on && d_prop_w.p, "DN_RUN_LEARNED needs dn_batch_set_proposal_net");
    DN_CHECK(patch == 7, "the learned initialisation uses the 7 x 7 patch");
    dn::LaunchArgs a = args(false);
    for (const SweepRange& r : sweep_ranges) {
      a.tiles = d_tiles_prop.p + r.first;
      a.n_tiles = r.count;
      DN_CUDA(dn::launch_sweep(a, d_feat.p, -1, prop_planes, r.S, stream));
    }
    for (const PropGroup& g : prop_groups) {
      const long long n_pix = (long long)g.n * g.W * g.H;
      const __nv_bfloat16* x = d_feat.p + g.off * dn::kFeatC;
      for (int k = 0; k < kPropLayers; ++k) {
        const bool last = k == kPropLayers - 1;
        __nv_bfloat16* y = (k & 1) ? d_act1.p : d_act0.p;
        dn::ConvArgs c{};
        c.x = x;
        c.w = d_prop_w.p + (size_t)k * 32 * 9 * 32;
        c.bias = d_prop_b.p + 32 * k;
        c.n_pix = n_pix;
        c.H = g.H;
        c.W = g.W;
        c.cin = 32;
        c.cout = last ? 4 : 32;
        c.relu = last ? 0 : 1;
        c.y = last ? nullptr : y + g.off * dn::kFeatC;
        c.y32 = last ? d_prop_out.p + 4 * g.off : nullptr;
        DN_CUDA(dn::conv3x3_forward(c, stream));
        x = c.y;
      }
    }
    DN_CUDA(dn::launch_proposal_to_planes(d_prop_out.p, d_maps.p, (int)maps.size(),
                                          prop_max_pixels, stream));
    return DN_OK;
  }

  // Enqueues the whole computation for every map on `stream`.
  // With the persistent launch the cleaner (with_clean) and the pruner
  // (with_prune) run inside it and tail_done is set; otherwise the caller
  // enqueues them after.
  bool tail_done = false;
  dn_status enqueue(Mode mode, bool timing = false, bool learned = false, bool with_clean = false,
                    bool with_prune = false) {
    tail_done = false;
    for (auto& m : maps) {
      const View& r = *views[m->ref];
      const size_t npx = (size_t)r.W * r.H;
      if (mode != Mode::kScorePlanes) {
        DN_CUDA(cudaMemsetAsync(m->state.p, 0, npx * sizeof(float4), stream));
        DN_CUDA(cudaMemsetAsync(m->score.p, 0, npx * sizeof(float), stream));
        DN_CUDA(cudaMemsetAsync(m->nghbr.p, 0, npx * sizeof(int), stream));
        if (active) DN_CUDA(cudaMemsetAsync(m->changed.p, 0, npx, stream));
      }
    }
    DN_CUDA(cudaMemsetAsync(d_taps.p, 0, 4 * sizeof(unsigned long long), stream));
    DN_CUDA(cudaMemsetAsync(d_error.p, 0, sizeof(int), stream));
    DN_TRY(mark(0, timing));
    timed_learned = learned && timing;
    if (learned) {
      DN_TRY(enqueue_proposal());
      DN_TRY(mark(7, timing));
    }
    dn::LaunchArgs a1 = args(false);
    a1.p.learned = learned ? 1 : 0;
    if (mode == Mode::kScorePlanes) {
      DN_CUDA(dn::launch_stage(dn::Stage::kScorePlanes, false, a1, stream));
      return DN_OK;
    }
    if (mode == Mode::kBruteForce) {
      DN_CUDA(dn::launch_stage(dn::Stage::kBruteForce, false, a1, stream));
      a1.flag = 0;
      DN_CUDA(dn::launch_stage(dn::Stage::kPostProcess, false, a1, stream));
      return DN_OK;
    }
    // Sample mode (ComputePatchMatchSample): the mode itself, or candidate
    // view mode 2; mode 1 keeps the full initialisation and scores one view
    // per candidate in the half-passes (dn_batch_set_candidate_views).
    const bool sample = (mode == Mode::kPatchMatchSample) || sample_hp == 2;
    const bool sample_half = sample || sample_hp;
    const int hp = half_passes >= 0 ? half_passes : 2 * iterations;
    if (persistent && !sample_half && patch == 7) {
      const int n_sync = dn::kPersistentCounters + hp;
      DN_CHECK(d_sync.p && d_sync.n >= (size_t)n_sync, "persistent launch buffers not prepared");
      DN_CUDA(cudaMemsetAsync(d_sync.p, 0, n_sync * sizeof(unsigned), stream));
      dn::PersistentArgs pa{};
      pa.base = a1;
      pa.tiles_init = d_tiles_init.p;
      pa.n_init = n_tiles_init;
      pa.tiles_hp = d_tiles2.p;
      pa.n_hp = n_tiles2;
      pa.tiles_post = d_tiles1.p;
      pa.n_post = n_tiles1;
      pa.n_half = hp;
      pa.sync = d_sync.p;
      pa.base.p.taps = d_taps.p + 1;
      if (with_clean) {
        pa.tail.clean_views = d_clean_views.p;
        pa.tail.cmaps = d_clean_maps.p;
        pa.tail.lists = d_clean_lists.p;
        pa.tail.clean_tiles = d_clean_tiles.p;
        pa.tail.n_clean = n_clean_tiles;
        pa.tail.min_views = min_consistent;
        pa.tail.thr = same_depth_thr;
      }
      if (with_clean && with_prune) {
        pa.tail.pmaps = d_prune_maps.p;
        pa.tail.n_pmaps = (int)maps.size();
        pa.tail.prune_tiles = d_prune_tiles.p;
        pa.tail.n_prune = n_prune_tiles;
      }
      tail_done = with_clean;
      DN_CUDA(dn::launch_persistent(pa, stream));
      DN_TRY(mark(1, timing));
      DN_TRY(mark(2, timing));
      DN_TRY(mark(3, timing));
      DN_TRY(mark(4, timing));
      return DN_OK;
    }
    dn::LaunchArgs ai = a1;
    ai.tiles = d_tiles_init.p;
    ai.n_tiles = n_tiles_init;
    DN_CUDA(dn::launch_stage(dn::Stage::kInit, sample, ai, stream));
    DN_TRY(mark(1, timing));
    dn::LaunchArgs a2 = args(true);
    a2.p.taps = d_taps.p + 1;
    for (int k = 0; k < hp; ++k) {
      a2.p.colour = k & 1;
      a2.p.pass = k;
      if (active && active_lists && k >= a2.p.active_from) {
        DN_CUDA(dn::launch_halfpass_list(sample_half, a2, (int)maps.size(), d_chunk0.p,
                                         d_tile_count.p, d_tile_off.p, stream));
      } else {
        DN_CUDA(dn::launch_stage(dn::Stage::kHalfPass, sample_half, a2, stream));
      }
    }
    DN_TRY(mark(2, timing));
    a1.flag = 1;
    DN_CUDA(dn::launch_stage(dn::Stage::kPostProcess, false, a1, stream));
    DN_TRY(mark(3, timing));
    DN_TRY(mark(4, timing));
    return DN_OK;
  }

  // Uploads the cleaner tables (outside any stream capture): one CleanView
  // per map (its final depth with its reference camera) and per map the
  // list of other maps it is checked against.
  dn_status prepare_clean() {
    std::vector<dn::CleanView> cv(maps.size());
    std::vector<dn::CleanMap> cmaps;
    std::vector<int4> tiles;
    std::vector<int> lists;
    for (size_t k = 0; k < maps.size(); ++k) {
      Map& m = *maps[k];
      const View& r = *views[m.ref];
      DN_CUDA(m.clean.alloc((size_t)r.W * r.H));
      dn::CleanView c{};
      c.depth = m.depth.p;
      c.W = r.W;
      c.H = r.H;
      c.stride = r.W;
      std::memcpy(c.K, r.cam.K, sizeof(c.K));
      std::memcpy(c.R, r.cam.R, sizeof(c.R));
      std::memcpy(c.t, r.cam.t, sizeof(c.t));
      cv[k] = c;
      dn::CleanMap cm{};
      cm.list_off = (int)lists.size();
      cm.n = (int)m.clean_maps.size();
      cm.out = m.clean.p;
      cmaps.push_back(cm);
      for (int o : m.clean_maps) lists.push_back(o);
      for (int y = 0; y < (r.H + dn::kCleanTileY - 1) / dn::kCleanTileY; ++y)
        for (int x = 0; x < (r.W + dn::kCleanTileX - 1) / dn::kCleanTileX; ++x)
          tiles.push_back(make_int4((int)k, x, y, 0));
    }
    DN_CUDA(d_clean_views.alloc(std::max<size_t>(cv.size(), 1)));
    DN_CUDA(d_clean_lists.alloc(std::max<size_t>(lists.size(), 1)));
    DN_CUDA(d_clean_maps.alloc(std::max<size_t>(cmaps.size(), 1)));
    DN_CUDA(d_clean_tiles.alloc(std::max<size_t>(tiles.size(), 1)));
    DN_CUDA(cudaMemcpyAsync(d_clean_views.p, cv.data(), cv.size() * sizeof(dn::CleanView),
                            cudaMemcpyHostToDevice, stream));
    if (!lists.empty())
      DN_CUDA(cudaMemcpyAsync(d_clean_lists.p, lists.data(), lists.size() * sizeof(int),
                              cudaMemcpyHostToDevice, stream));
    DN_CUDA(cudaMemcpyAsync(d_clean_maps.p, cmaps.data(), cmaps.size() * sizeof(dn::CleanMap),
                            cudaMemcpyHostToDevice, stream));
    DN_CUDA(cudaMemcpyAsync(d_clean_tiles.p, tiles.data(), tiles.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, stream));
    n_clean_tiles = (int)tiles.size();
    DN_CUDA(cudaStreamSynchronize(stream));
    return DN_OK;
  }
  DevBuf<dn::CleanMap> d_clean_maps;
  DevBuf<int4> d_clean_tiles;
  int n_clean_tiles = 0;

  // Pruner tables and buffers (outside any stream capture): per map the
  // cleaned depth and PatchMatch planes of the map and its cleaner maps.
  DevBuf<unsigned long long> d_prune_counts;
  DevBuf<dn::PruneMap> d_prune_maps;
  DevBuf<int4> d_prune_tiles;
  int n_prune_tiles = 0;
  dn_status prepare_prune() {
    DN_CUDA(d_prune_counts.alloc(std::max<size_t>(maps.size(), 1)));
    std::vector<dn::PruneMap> pmaps;
    std::vector<int4> tiles;
    for (size_t k = 0; k < maps.size(); ++k) {
      Map& m = *maps[k];
      const View& r = *views[m.ref];
      const size_t npx = (size_t)r.W * r.H;
      std::vector<dn::PruneView> pv;
      std::vector<int> ids = {(int)k};
      for (int o : m.clean_maps) ids.push_back(o);
      for (int id : ids) {
        Map& om = *maps[id];
        const View& ov = *views[om.ref];
        dn::PruneView v{};
        v.depth = om.clean.p;
        v.plane = reinterpret_cast<const float*>(om.state.p);
        v.plane_stride = 4;
        v.color = nullptr;
        v.label = nullptr;
        v.gray = ov.gray.p;
        v.W = ov.W;
        v.H = ov.H;
        std::memcpy(v.K, ov.cam.K, sizeof(v.K));
        std::memcpy(v.R, ov.cam.R, sizeof(v.R));
        std::memcpy(v.t, ov.cam.t, sizeof(v.t));
        pv.push_back(v);
      }
      DN_CUDA(m.prune_views.alloc(pv.size()));
      DN_CUDA(m.prune_scratch.alloc(dn::prune_batch_scratch_bytes(r.W, r.H)));
      DN_CUDA(m.prune_points.alloc(3 * npx));
      DN_CUDA(m.prune_normals.alloc(3 * npx));
      DN_CUDA(m.prune_colors.alloc(3 * npx));
      DN_CUDA(m.prune_labels.alloc(npx));
      DN_CUDA(cudaMemcpyAsync(m.prune_views.p, pv.data(), pv.size() * sizeof(dn::PruneView),
                              cudaMemcpyHostToDevice, stream));
      const dn::PruneOut o{m.prune_points.p, m.prune_normals.p, m.prune_colors.p,
                           m.prune_labels.p};
      pmaps.push_back(dn::prune_batch_map(m.prune_views.p, (int)pv.size(), r.W, r.H,
                                          m.prune_scratch.p, o, d_prune_counts.p + k));
      for (int blk = 0; blk < pmaps.back().blocks; ++blk)
        tiles.push_back(make_int4((int)k, blk, 0, 0));
    }
    DN_CUDA(d_prune_maps.alloc(std::max<size_t>(pmaps.size(), 1)));
    DN_CUDA(d_prune_tiles.alloc(std::max<size_t>(tiles.size(), 1)));
    DN_CUDA(cudaMemcpyAsync(d_prune_maps.p, pmaps.data(), pmaps.size() * sizeof(dn::PruneMap),
                            cudaMemcpyHostToDevice, stream));
    DN_CUDA(cudaMemcpyAsync(d_prune_tiles.p, tiles.data(), tiles.size() * sizeof(int4),
                            cudaMemcpyHostToDevice, stream));
    n_prune_tiles = (int)tiles.size();
    DN_CUDA(cudaStreamSynchronize(stream));
    return DN_OK;
  }
  // The pruner over every map in three launches (flags, per-map scans,
  // ordered writes).
  dn_status enqueue_prune() {
    DN_CUDA(dn::launch_prune_batch(d_prune_maps.p, (int)maps.size(), d_prune_tiles.p,
                                   n_prune_tiles, same_depth_thr, stream));
    DN_TRY(mark(4, timed));
    return DN_OK;
  }

  // The cleaner over every map in one launch.
  dn_status enqueue_clean(bool timing = false) {
    DN_CUDA(dn::launch_clean_batch(d_clean_views.p, d_clean_maps.p, d_clean_lists.p,
                                   d_clean_tiles.p, n_clean_tiles, same_depth_thr, min_consistent,
                                   stream));
    DN_TRY(mark(4, timing));
    return DN_OK;
  }

  dn_status set_view_image(int v, const uint8_t* image, int stride) {
    DN_CHECK(v >= 0 && v < (int)views.size(), "view id out of range");
    DN_CHECK(image, "image must not be NULL");
    View& w = *views[v];
    if (stride <= 0) stride = w.W;
    DN_CHECK(stride >= w.W, "stride must be >= width");
    DN_CUDA(cudaSetDevice(device));
    DN_TRY(flush_uploads());  // an earlier pipelined upload of the view must not win
    const dn::TableGeom tg = dn::table_geom(w.W, w.H);
    DN_CUDA(cudaMemcpy2DAsync(w.gray.p, w.W, image, stride, w.W, w.H, cudaMemcpyHostToDevice, stream));
    DN_CUDA(dn::launch_prepare_view(w.gray.p, w.W, w.H, w.W, w.img.p, w.quad.p, tg.TP, tg.TW, tg.TH,
                                    w.cbias, stream));
    return DN_OK;
  }

  // The same replacement, pipelined: the host copy runs on the upload stream
  // while earlier batch-stream work (a run) is still executing.  The view's
  // FP16 image and coefficient table are rebuilt by the next work on the
  // batch stream that reads views, for every uploaded view at once.
  dn_status upload_view_image(int v, const uint8_t* image, int stride) {
    DN_CHECK(v >= 0 && v < (int)views.size(), "view id out of range");
    DN_CHECK(image, "image must not be NULL");
    View& w = *views[v];
    if (stride <= 0) stride = w.W;
    DN_CHECK(stride >= w.W, "stride must be >= width");
    DN_CUDA(cudaSetDevice(device));
    DN_CUDA(w.upload.alloc((size_t)w.W * w.H));
    // The last flush has read every upload buffer.
    DN_CUDA(cudaStreamWaitEvent(up, ev_consumed, 0));
    DN_CUDA(cudaMemcpy2DAsync(w.upload.p, w.W, image, stride, w.W, w.H, cudaMemcpyHostToDevice, up));
    if (std::find(pending_uploads.begin(), pending_uploads.end(), v) == pending_uploads.end())
      pending_uploads.push_back(v);
    return DN_OK;
  }

  dn_status timings(float* out, int n, uint64_t* taps_out) {
    DN_CHECK(out || n == 0, "NULL output");
    DN_CHECK(timed, "the last run was not made with DN_RUN_TIMING");
    DN_CUDA(cudaSetDevice(device));
    DN_CUDA(cudaStreamSynchronize(stream));
    float t[6] = {0, 0, 0, 0, 0, 0};
    // With the learned proposal, init starts at its end event (7).
    DN_CUDA(cudaEventElapsedTime(&t[0], ev[timed_learned ? 7 : 0], ev[1]));
    DN_CUDA(cudaEventElapsedTime(&t[1], ev[1], ev[2]));
    DN_CUDA(cudaEventElapsedTime(&t[2], ev[2], ev[3]));
    DN_CUDA(cudaEventElapsedTime(&t[3], ev[3], ev[4]));
    DN_CUDA(cudaEventElapsedTime(&t[4], ev[0], ev[4]));
    if (timed_learned) DN_CUDA(cudaEventElapsedTime(&t[5], ev[0], ev[7]));
    for (int k = 0; k < n && k < 6; ++k) out[k] = t[k];
    if (taps_out) {
      unsigned long long v[4];
      DN_CUDA(cudaMemcpy(v, d_taps.p, sizeof(v), cudaMemcpyDeviceToHost));
      taps_out[0] = v[0];
      taps_out[1] = v[1];
    }
    return DN_OK;
  }

  dn_status finish() {
    DN_CUDA(cudaStreamSynchronize(stream));
    DN_CUDA(cudaStreamSynchronize(up));
    DN_CUDA(cudaStreamSynchronize(down));
    int err = 0;
    DN_CUDA(cudaMemcpy(&err, d_error.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(DN_TIMEOUT, "a bounded device-side wait expired");
    if (prop_on && dn::take_tc_error() != 0)
      return fail(DN_TIMEOUT, "a bounded wait of the proposal network expired");
    computed = true;
    return DN_OK;
  }

  dn_status compute(Mode mode) {
    DN_CUDA(cudaSetDevice(device));
    DN_TRY(check_params(mode));
    DN_TRY(prepare());
    DN_TRY(enqueue(mode));
    return finish();
  }

  dn_status fetch(int map, float* depth, float* plane, float* score, int32_t* nghbr,
                  float* clean) {
    DN_CHECK(map >= 0 && map < (int)maps.size(), "depthmap id out of range");
    DN_CHECK(computed, "no result computed yet");
    DN_CUDA(cudaSetDevice(device));
    Map& m = *maps[map];
    const View& r = *views[m.ref];
    const size_t npx = (size_t)r.W * r.H;
    if (depth)
      DN_CUDA(cudaMemcpyAsync(depth, m.depth.p, npx * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (plane) {
      DN_CUDA(m.plane_out.alloc(3 * npx));
      DN_CUDA(dn::launch_pack(d_maps.p, map, m.plane_out.p, npx, stream));
      DN_CUDA(cudaMemcpyAsync(plane, m.plane_out.p, 3 * npx * sizeof(float),
                              cudaMemcpyDeviceToHost, stream));
    }
    if (score)
      DN_CUDA(cudaMemcpyAsync(score, m.score.p, npx * sizeof(float), cudaMemcpyDeviceToHost, stream));
    if (nghbr)
      DN_CUDA(cudaMemcpyAsync(nghbr, m.nghbr.p, npx * sizeof(int), cudaMemcpyDeviceToHost, stream));
    if (clean) {
      DN_CHECK(m.clean.p, "the depthmap was not cleaned");
      DN_CUDA(cudaMemcpyAsync(clean, m.clean.p, npx * sizeof(float), cudaMemcpyDeviceToHost, stream));
    }
    DN_CUDA(cudaStreamSynchronize(stream));
    return DN_OK;
  }

  // Final depths of several maps into host buffers: every copy is queued on
  // the batch stream (asynchronous for pinned buffers), one synchronisation.
  dn_status fetch_depths(int n, const int* ids, float* const* outs, int clean) {
    DN_CHECK(n >= 0 && (n == 0 || (ids && outs)), "NULL argument");
    DN_CHECK(computed, "no result computed yet");
    DN_CUDA(cudaSetDevice(device));
    for (int k = 0; k < n; ++k) {
      DN_CHECK(ids[k] >= 0 && ids[k] < (int)maps.size(), "depthmap id out of range");
      DN_CHECK(outs[k], "NULL output buffer");
      const Map& m = *maps[ids[k]];
      DN_CHECK(!clean || m.clean.p, "the depthmap was not cleaned");
    }
    for (int k = 0; k < n; ++k) {
      const Map& m = *maps[ids[k]];
      const View& r = *views[m.ref];
      DN_CUDA(cudaMemcpyAsync(outs[k], clean ? m.clean.p : m.depth.p,
                              (size_t)r.W * r.H * sizeof(float), cudaMemcpyDeviceToHost, stream));
    }
    DN_CUDA(cudaStreamSynchronize(stream));
    return DN_OK;
  }

  // The same readback, pipelined: the depths as the batch stream leaves them
  // at this point are gathered into a staging buffer on the batch stream (one
  // launch), then copied to the host on the readback stream, so a run enqueued
  // next overlaps the host copies.  Two staging buffers alternate; a third
  // readback in flight waits for the first one's host copies.
  dn_status fetch_depths_async(int n, const int* ids, float* const* outs, int clean) {
    DN_CHECK(n >= 0 && (n == 0 || (ids && outs)), "NULL argument");
    DN_CHECK(computed, "no result computed yet");
    DN_CUDA(cudaSetDevice(device));
    std::vector<const float*> src(n);
    std::vector<size_t> count(n), off(n);
    size_t total = 0;
    for (int k = 0; k < n; ++k) {
      DN_CHECK(ids[k] >= 0 && ids[k] < (int)maps.size(), "depthmap id out of range");
      DN_CHECK(outs[k], "NULL output buffer");
      const Map& m = *maps[ids[k]];
      DN_CHECK(!clean || m.clean.p, "the depthmap was not cleaned");
      src[k] = clean ? m.clean.p : m.depth.p;
      count[k] = (size_t)views[m.ref]->W * views[m.ref]->H;
      off[k] = total;
      total += (count[k] + 3) & ~(size_t)3;  // 16-byte aligned arrays
    }
    if (n == 0) return DN_OK;
    const int s = stage_next;
    stage_next ^= 1;
    DevBuf<float>& st = d_stage[s];
    if (st.n < total) {
      DN_CUDA(cudaEventSynchronize(ev_stage_done[s]));
      DN_CUDA(st.alloc(total));
    }
    DN_CUDA(cudaStreamWaitEvent(stream, ev_stage_done[s], 0));
    DN_CUDA(dn::launch_gather_floats(src.data(), count.data(), off.data(), n, st.p, stream));
    DN_CUDA(cudaEventRecord(ev_staged, stream));
    DN_CUDA(cudaStreamWaitEvent(down, ev_staged, 0));
    for (int k = 0; k < n; ++k)
      DN_CUDA(cudaMemcpyAsync(outs[k], st.p + off[k], count[k] * sizeof(float),
                              cudaMemcpyDeviceToHost, down));
    DN_CUDA(cudaEventRecord(ev_stage_done[s], down));
    return DN_OK;
  }

  dn_status set_init(int map, const float* planes) {
    DN_CHECK(map >= 0 && map < (int)maps.size(), "depthmap id out of range");
    Map& m = *maps[map];
    const View& r = *views[m.ref];
    const size_t npx = (size_t)r.W * r.H;
    DN_CUDA(cudaSetDevice(device));
    if (!planes) {
      m.has_init = false;
      invalidate();
      return DN_OK;
    }
    const bool had = m.has_init;
    DN_CUDA(m.init.alloc(3 * npx));
    DN_CUDA(cudaMemcpyAsync(m.init.p, planes, 3 * npx * sizeof(float), cudaMemcpyHostToDevice, stream));
    DN_CUDA(cudaStreamSynchronize(stream));
    m.has_init = true;
    if (!had) invalidate();
    return DN_OK;
  }

  dn_status taps(uint64_t* out) {
    DN_CHECK(out, "NULL output");
    DN_CUDA(cudaSetDevice(device));
    unsigned long long v[4] = {0, 0, 0, 0};
    DN_CUDA(cudaMemcpy(v, d_taps.p, sizeof(v), cudaMemcpyDeviceToHost));
    *out = v[0] + v[1] + v[2] + v[3];
    return DN_OK;
  }
};

}  // namespace

// ======================================================================
// C ABI

struct dn_estimator {
  Engine eng;
  int W = 0, H = 0;
  double min_d = 0, max_d = 0;
};

struct dn_cleaner {
  int device = 0;
  cudaStream_t stream = nullptr;
  float thr = 0.01f;
  int min_views = 2;
  std::vector<dn::CleanView> views;
  std::vector<DevBuf<float>> depths;
  DevBuf<dn::CleanView> d_views;
  DevBuf<int> d_others;
  DevBuf<float> d_out;
  ~dn_cleaner() {
    if (stream) cudaStreamDestroy(stream);
  }
};

struct dn_gpu_cleaner {
  int device = 0;
  cudaStream_t stream = nullptr;
  float thr = 0.01f;
  int min_views = 3;
  float carving = 0.2f;
  int max_carved = 1;
  struct V {
    dn::GpuCleanCam cam;
    int W, H;
    DevBuf<float> depth;
  };
  std::vector<V> views;
  DevBuf<float> d_out;
  ~dn_gpu_cleaner() {
    if (stream) cudaStreamDestroy(stream);
  }
};

struct dn_pruner {
  int device = 0;
  cudaStream_t stream = nullptr;
  float thr = 0.01f;
  std::vector<dn::PruneView> views;
  std::vector<DevBuf<float>> depths, planes;
  std::vector<DevBuf<uint8_t>> colors, labels;
  DevBuf<dn::PruneView> d_views;
  DevBuf<uint8_t> scratch;
  DevBuf<float> points, normals;
  DevBuf<uint8_t> out_colors, out_labels;
  DevBuf<unsigned long long> d_count;
  int64_t count = -1;
  ~dn_pruner() {
    if (stream) cudaStreamDestroy(stream);
  }
};

struct dn_batch {
  Engine eng;
  bool ran = false;
};

extern "C" {

const char* dn_last_error(void) { return g_last_error.c_str(); }
const char* dn_version(void) { return "opensfm_b200 dense 0.1 (sm_100a)"; }
int dn_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

dn_status dn_set_device(int device) {
  DN_CHECK(device >= 0 && device < dn_device_count(), "device index out of range");
  DN_CUDA(cudaSetDevice(device));
  return DN_OK;
}

static dn_status need_device() {
  if (dn_device_count() <= 0) return fail(DN_DEVICE_ERROR, "no CUDA device available");
  return DN_OK;
}

// ------------------------------------------------------------- estimator
dn_status dn_estimator_create(dn_estimator** out) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(out, "NULL output");
  *out = nullptr;
  DN_TRY(need_device());
  auto e = std::make_unique<dn_estimator>();
  DN_TRY(e->eng.init());
  *out = e.release();
  return DN_OK;
}

dn_status dn_estimator_destroy(dn_estimator* est) {
  const dn::DeviceRestore device_restore_;
  delete est;
  return DN_OK;
}

dn_status dn_estimator_add_view(dn_estimator* est, const double* K, const double* R,
                                const double* t, const uint8_t* image, const uint8_t* mask,
                                int width, int height, int stride) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(est, "NULL estimator");
  DN_CHECK((int)est->eng.views.size() <= dn::kMaxNbr, "at most 17 views (reference + 16)");
  int id;
  DN_TRY(est->eng.add_view(K, R, t, image, mask, width, height, stride, &id));
  if (id == 0) {
    est->W = width;
    est->H = height;
  }
  // One depthmap: view 0 against every other view.
  est->eng.maps.clear();
  if (est->eng.views.size() >= 2) {
    std::vector<int> nb;
    for (int k = 1; k < (int)est->eng.views.size(); ++k) nb.push_back(k);
    DN_TRY(est->eng.add_map(0, nb.data(), (int)nb.size(), est->min_d, est->max_d, nullptr));
  }
  return DN_OK;
}

dn_status dn_estimator_set_depth_range(dn_estimator* est, double mn, double mx, int n) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(est, "NULL estimator");
  est->min_d = mn;
  est->max_d = mx;
  est->eng.num_planes = n;
  for (auto& m : est->eng.maps) {
    m->min_d = mn;
    m->max_d = mx;
  }
  est->eng.invalidate();
  return DN_OK;
}

dn_status dn_estimator_set_patchmatch_iterations(dn_estimator* est, int n) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(est, "NULL estimator");
  est->eng.iterations = n;
  est->eng.invalidate();
  return DN_OK;
}

dn_status dn_estimator_set_patch_size(dn_estimator* est, int size) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(est, "NULL estimator");
  const int hpz = (size - 1) / 2;
  DN_CHECK(hpz >= 1 && hpz <= dn::kMaxHpz, "patch size must be in 3..12");
  est->eng.patch = size;
  return DN_OK;
}

dn_status dn_estimator_set_min_patch_sd(dn_estimator* est, float sd) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(est, "NULL estimator");
  est->eng.min_var = sd * sd;
  return DN_OK;
}

dn_status dn_estimator_set_seed(dn_estimator* est, uint64_t seed) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(est, "NULL estimator");
  est->eng.seed = seed;
  return DN_OK;
}

static dn_status est_compute(dn_estimator* est, Mode mode, float* depth, float* plane,
                             float* score, int32_t* nghbr) {
  DN_CHECK(est, "NULL estimator");
  DN_CHECK(est->eng.views.size() >= 2, "DepthmapEstimator needs a reference and at least one other view");
  DN_CHECK(depth && plane && score && nghbr, "output buffers must not be NULL");
  DN_TRY(est->eng.compute(mode));
  return est->eng.fetch(0, depth, plane, score, nghbr, nullptr);
}

dn_status dn_estimator_compute_brute_force(dn_estimator* est, float* depth, float* plane,
                                           float* score, int32_t* nghbr) {
  const dn::DeviceRestore device_restore_;
  if (est && est->eng.maps.size() == 1 && est->eng.maps[0]->has_init) est->eng.set_init(0, nullptr);
  return est_compute(est, Mode::kBruteForce, depth, plane, score, nghbr);
}

dn_status dn_estimator_compute_patch_match(dn_estimator* est, float* depth, float* plane,
                                           float* score, int32_t* nghbr) {
  const dn::DeviceRestore device_restore_;
  if (est && est->eng.maps.size() == 1 && est->eng.maps[0]->has_init) est->eng.set_init(0, nullptr);
  return est_compute(est, Mode::kPatchMatch, depth, plane, score, nghbr);
}

dn_status dn_estimator_compute_patch_match_sample(dn_estimator* est, float* depth,
                                                  float* plane, float* score, int32_t* nghbr) {
  const dn::DeviceRestore device_restore_;
  if (est && est->eng.maps.size() == 1 && est->eng.maps[0]->has_init) est->eng.set_init(0, nullptr);
  return est_compute(est, Mode::kPatchMatchSample, depth, plane, score, nghbr);
}

dn_status dn_estimator_compute_patch_match_init(dn_estimator* est, const float* init_planes,
                                                float* depth, float* plane, float* score,
                                                int32_t* nghbr) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(est, "NULL estimator");
  DN_CHECK(init_planes, "init planes must not be NULL");
  DN_CHECK(est->eng.maps.size() == 1, "DepthmapEstimator needs a reference and at least one other view");
  DN_TRY(est->eng.set_init(0, init_planes));
  return est_compute(est, Mode::kPatchMatch, depth, plane, score, nghbr);
}

dn_status dn_estimator_score_planes(dn_estimator* est, const float* planes, float* score,
                                    int32_t* nghbr) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(est, "NULL estimator");
  DN_CHECK(planes && score && nghbr, "buffers must not be NULL");
  DN_CHECK(est->eng.views.size() >= 2, "DepthmapEstimator needs a reference and at least one other view");
  DN_TRY(est->eng.set_init(0, planes));
  DN_TRY(est->eng.compute(Mode::kScorePlanes));
  dn_status s = est->eng.fetch(0, nullptr, nullptr, score, nghbr, nullptr);
  est->eng.set_init(0, nullptr);
  return s;
}

dn_status dn_estimator_last_taps(dn_estimator* est, uint64_t* taps) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(est, "NULL estimator");
  return est->eng.taps(taps);
}

// ---------------------------------------------------------------- cleaner
// ------------------------------------------------------- GPUDepthmapCleaner
dn_status dn_gpu_cleaner_create(dn_gpu_cleaner** out) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(out, "NULL output");
  *out = nullptr;
  DN_TRY(need_device());
  auto c = std::make_unique<dn_gpu_cleaner>();
  DN_CUDA(cudaGetDevice(&c->device));
  DN_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  *out = c.release();
  return DN_OK;
}
dn_status dn_gpu_cleaner_destroy(dn_gpu_cleaner* c) {
  const dn::DeviceRestore device_restore_;
  delete c;
  return DN_OK;
}
dn_status dn_gpu_cleaner_set_same_depth_threshold(dn_gpu_cleaner* c, float t) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  c->thr = t;
  return DN_OK;
}
dn_status dn_gpu_cleaner_set_min_consistent_views(dn_gpu_cleaner* c, int n) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  c->min_views = n;
  return DN_OK;
}
dn_status dn_gpu_cleaner_set_carving_threshold(dn_gpu_cleaner* c, float t) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  c->carving = std::max(0.0f, t);  // cleaner.cc:31-33
  return DN_OK;
}
dn_status dn_gpu_cleaner_set_max_carved_views(dn_gpu_cleaner* c, int n) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  c->max_carved = std::max(0, n);  // cleaner.cc:35-37
  return DN_OK;
}
dn_status dn_gpu_cleaner_set_device(dn_gpu_cleaner* c, int device) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  DN_CHECK(device >= 0 && device < dn_device_count(), "device index out of range");
  DN_CHECK(c->views.empty(), "set_device must come before the first add_view");
  if (device == c->device) return DN_OK;
  DN_CUDA(cudaSetDevice(c->device));
  c->d_out.release();
  if (c->stream) DN_CUDA(cudaStreamDestroy(c->stream));
  c->stream = nullptr;
  DN_CUDA(cudaSetDevice(device));
  DN_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  c->device = device;
  return DN_OK;
}
dn_status dn_gpu_cleaner_add_view(dn_gpu_cleaner* c, const double* K, const double* R,
                                  const double* t, const float* depth, int width, int height,
                                  int stride, int* id) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  DN_TRY(check_camera(K, R, t));
  DN_CHECK(depth, "depth must not be NULL");
  DN_CHECK(width >= 2 && height >= 2 && width <= 16384 && height <= 16384, "bad depthmap size");
  if (stride <= 0) stride = width;
  DN_CHECK(stride >= width, "stride must be >= width");
  DN_CUDA(cudaSetDevice(c->device));
  dn_gpu_cleaner::V v;
  DN_CUDA(v.depth.alloc((size_t)width * height));
  DN_CUDA(cudaMemcpy2DAsync(v.depth.p, width * sizeof(float), depth, stride * sizeof(float),
                            width * sizeof(float), height, cudaMemcpyHostToDevice, c->stream));
  DN_CUDA(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 9; ++k) {
    v.cam.K[k] = (float)K[k];  // opencl_utils.h:238-252 casts the camera to FP32
    v.cam.R[k] = (float)R[k];
  }
  for (int k = 0; k < 3; ++k) v.cam.t[k] = (float)t[k];
  v.W = width;
  v.H = height;
  c->views.push_back(std::move(v));
  if (id) *id = (int)c->views.size() - 1;
  return DN_OK;
}
dn_status dn_gpu_cleaner_clean(dn_gpu_cleaner* c, int ref, const int* neighbor_ids, int n,
                               float* out) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c && out, "NULL argument");
  DN_CHECK(n >= 0 && (n == 0 || neighbor_ids), "NULL neighbour list");
  const int nv = (int)c->views.size();
  if (ref < 0 || ref >= nv) {
    g_last_error = "Clean: ref_idx out of range";
    return DN_OUT_OF_RANGE;
  }
  for (int k = 0; k < n; ++k)
    if (neighbor_ids[k] < 0 || neighbor_ids[k] >= nv) {
      g_last_error = "Clean: neighbor id out of range";
      return DN_OUT_OF_RANGE;
    }
  const auto& r = c->views[ref];
  const int n_src = std::min(n, dn::kMaxGpuCleanSources);
  dn::GpuCleanArgs a{};
  a.ref = r.depth.p;
  a.W = r.W;
  a.H = r.H;
  a.cam[0] = r.cam;
  for (int k = 0; k < n_src; ++k) {
    const auto& o = c->views[neighbor_ids[k]];
    // The reference resizes a source of another size to the reference's but
    // keeps its intrinsics (cleaner.cc:115-134); only equal sizes are taken.
    DN_CHECK(o.W == r.W && o.H == r.H, "every source depthmap must have the reference's size");
    a.src[k] = o.depth.p;
    a.cam[k + 1] = o.cam;
  }
  a.n_src = n_src;
  a.same_depth_threshold = c->thr;
  a.min_consistent = std::min(c->min_views, 1 + n);  // effective_min, cleaner.cc:148
  a.carving_threshold = c->carving;
  a.max_carved = c->max_carved;
  DN_CUDA(cudaSetDevice(c->device));
  const size_t npx = (size_t)r.W * r.H;
  if (c->d_out.n < npx) DN_CUDA(c->d_out.alloc(npx));
  DN_CUDA(dn::launch_gpu_clean(a, c->d_out.p, c->stream));
  DN_CUDA(cudaMemcpyAsync(out, c->d_out.p, npx * sizeof(float), cudaMemcpyDeviceToHost,
                          c->stream));
  DN_CUDA(cudaStreamSynchronize(c->stream));
  return DN_OK;
}
dn_status dn_gpu_cleaner_clear(dn_gpu_cleaner* c) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  c->views.clear();
  c->d_out.release();
  return DN_OK;
}

dn_status dn_cleaner_create(dn_cleaner** out) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(out, "NULL output");
  *out = nullptr;
  DN_TRY(need_device());
  auto c = std::make_unique<dn_cleaner>();
  DN_CUDA(cudaGetDevice(&c->device));
  DN_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  *out = c.release();
  return DN_OK;
}
dn_status dn_cleaner_destroy(dn_cleaner* c) {
  const dn::DeviceRestore device_restore_;
  delete c;
  return DN_OK;
}
dn_status dn_cleaner_set_same_depth_threshold(dn_cleaner* c, float t) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  c->thr = t;
  return DN_OK;
}
dn_status dn_cleaner_set_min_consistent_views(dn_cleaner* c, int n) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  c->min_views = n;
  return DN_OK;
}
dn_status dn_cleaner_add_view(dn_cleaner* c, const double* K, const double* R, const double* t,
                              const float* depth, int width, int height, int stride) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  DN_TRY(check_camera(K, R, t));
  DN_CHECK(depth, "depth must not be NULL");
  DN_CHECK(width >= 1 && height >= 1 && width <= 16384 && height <= 16384, "bad depthmap size");
  if (stride <= 0) stride = width;
  DN_CHECK(stride >= width, "stride must be >= width");
  DN_CUDA(cudaSetDevice(c->device));
  DevBuf<float> d;
  DN_CUDA(d.alloc((size_t)width * height));
  DN_CUDA(cudaMemcpy2DAsync(d.p, width * sizeof(float), depth, stride * sizeof(float),
                            width * sizeof(float), height, cudaMemcpyHostToDevice, c->stream));
  DN_CUDA(cudaStreamSynchronize(c->stream));
  dn::CleanView v{};
  v.depth = d.p;
  v.W = width;
  v.H = height;
  v.stride = width;
  std::memcpy(v.K, K, sizeof(v.K));
  std::memcpy(v.R, R, sizeof(v.R));
  std::memcpy(v.t, t, sizeof(v.t));
  c->views.push_back(v);
  c->depths.push_back(std::move(d));
  return DN_OK;
}
dn_status dn_cleaner_clean(dn_cleaner* c, float* clean_depth) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(c, "NULL cleaner");
  DN_CHECK(clean_depth, "output must not be NULL");
  DN_CHECK(!c->views.empty(), "DepthmapCleaner has no views");
  DN_CUDA(cudaSetDevice(c->device));
  const int W = c->views[0].W, H = c->views[0].H;
  const int n = (int)c->views.size();
  DN_CUDA(c->d_views.alloc(n));
  DN_CUDA(c->d_others.alloc(std::max(n - 1, 1)));
  DN_CUDA(c->d_out.alloc((size_t)W * H));
  std::vector<int> others;
  for (int k = 1; k < n; ++k) others.push_back(k);
  DN_CUDA(cudaMemcpyAsync(c->d_views.p, c->views.data(), n * sizeof(dn::CleanView),
                          cudaMemcpyHostToDevice, c->stream));
  if (!others.empty())
    DN_CUDA(cudaMemcpyAsync(c->d_others.p, others.data(), others.size() * sizeof(int),
                            cudaMemcpyHostToDevice, c->stream));
  DN_CUDA(dn::launch_clean(c->d_views.p, 0, c->d_others.p, n - 1, W, H, c->thr, c->min_views,
                           c->d_out.p, c->stream));
  DN_CUDA(cudaMemcpyAsync(clean_depth, c->d_out.p, (size_t)W * H * sizeof(float),
                          cudaMemcpyDeviceToHost, c->stream));
  DN_CUDA(cudaStreamSynchronize(c->stream));
  return DN_OK;
}

// ----------------------------------------------------------------- pruner
dn_status dn_pruner_create(dn_pruner** out) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(out, "NULL output");
  *out = nullptr;
  DN_TRY(need_device());
  auto p = std::make_unique<dn_pruner>();
  DN_CUDA(cudaGetDevice(&p->device));
  DN_CUDA(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
  DN_CUDA(p->d_count.alloc(1));
  *out = p.release();
  return DN_OK;
}
dn_status dn_pruner_destroy(dn_pruner* p) {
  const dn::DeviceRestore device_restore_;
  delete p;
  return DN_OK;
}
dn_status dn_pruner_set_same_depth_threshold(dn_pruner* p, float t) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(p, "NULL pruner");
  p->thr = t;
  return DN_OK;
}
dn_status dn_pruner_add_view(dn_pruner* p, const double* K, const double* R, const double* t,
                             const float* depth, const float* plane, const uint8_t* color,
                             const uint8_t* label, int width, int height) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(p, "NULL pruner");
  DN_TRY(check_camera(K, R, t));
  DN_CHECK(depth && plane && color && label, "depth, plane, color and label must not be NULL");
  DN_CHECK(width >= 1 && height >= 1 && width <= 16384 && height <= 16384, "bad depthmap size");
  DN_CUDA(cudaSetDevice(p->device));
  const size_t n = (size_t)width * height;
  DevBuf<float> d, pl;
  DevBuf<uint8_t> col, lab;
  DN_CUDA(d.alloc(n));
  DN_CUDA(pl.alloc(3 * n));
  DN_CUDA(col.alloc(3 * n));
  DN_CUDA(lab.alloc(n));
  DN_CUDA(cudaMemcpyAsync(d.p, depth, n * sizeof(float), cudaMemcpyHostToDevice, p->stream));
  DN_CUDA(cudaMemcpyAsync(pl.p, plane, 3 * n * sizeof(float), cudaMemcpyHostToDevice, p->stream));
  DN_CUDA(cudaMemcpyAsync(col.p, color, 3 * n, cudaMemcpyHostToDevice, p->stream));
  DN_CUDA(cudaMemcpyAsync(lab.p, label, n, cudaMemcpyHostToDevice, p->stream));
  DN_CUDA(cudaStreamSynchronize(p->stream));
  dn::PruneView v{};
  v.plane_stride = 3;
  v.depth = d.p;
  v.plane = pl.p;
  v.color = col.p;
  v.label = lab.p;
  v.W = width;
  v.H = height;
  std::memcpy(v.K, K, sizeof(v.K));
  std::memcpy(v.R, R, sizeof(v.R));
  std::memcpy(v.t, t, sizeof(v.t));
  p->views.push_back(v);
  p->depths.push_back(std::move(d));
  p->planes.push_back(std::move(pl));
  p->colors.push_back(std::move(col));
  p->labels.push_back(std::move(lab));
  p->count = -1;
  return DN_OK;
}
dn_status dn_pruner_prune(dn_pruner* p, int64_t* count) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(p, "NULL pruner");
  DN_CHECK(count, "NULL count");
  DN_CHECK(!p->views.empty(), "DepthmapPruner has no views");
  DN_CUDA(cudaSetDevice(p->device));
  const int W = p->views[0].W, H = p->views[0].H;
  const size_t n = (size_t)W * H;
  const int nv = (int)p->views.size();
  DN_CUDA(p->d_views.alloc(nv));
  DN_CUDA(p->scratch.alloc(dn::prune_scratch_bytes(W, H)));
  DN_CUDA(p->points.alloc(3 * n));
  DN_CUDA(p->normals.alloc(3 * n));
  DN_CUDA(p->out_colors.alloc(3 * n));
  DN_CUDA(p->out_labels.alloc(n));
  DN_CUDA(cudaMemcpyAsync(p->d_views.p, p->views.data(), nv * sizeof(dn::PruneView),
                          cudaMemcpyHostToDevice, p->stream));
  dn::PruneOut o{p->points.p, p->normals.p, p->out_colors.p, p->out_labels.p};
  DN_CUDA(dn::launch_prune(p->d_views.p, nv, W, H, p->thr, p->scratch.p, o, p->d_count.p,
                           p->stream));
  unsigned long long c = 0;
  DN_CUDA(cudaMemcpyAsync(&c, p->d_count.p, sizeof(c), cudaMemcpyDeviceToHost, p->stream));
  DN_CUDA(cudaStreamSynchronize(p->stream));
  p->count = (int64_t)c;
  *count = p->count;
  return DN_OK;
}
dn_status dn_pruner_fetch(dn_pruner* p, float* points, float* normals, uint8_t* colors,
                          uint8_t* labels, int64_t capacity) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(p, "NULL pruner");
  DN_CHECK(p->count >= 0, "dn_pruner_prune has not run since the last add_view");
  DN_CHECK(capacity >= p->count, "capacity is smaller than the pruned point count");
  DN_CUDA(cudaSetDevice(p->device));
  const size_t n = (size_t)p->count;
  if (n) {
    if (points)
      DN_CUDA(cudaMemcpyAsync(points, p->points.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, p->stream));
    if (normals)
      DN_CUDA(cudaMemcpyAsync(normals, p->normals.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost, p->stream));
    if (colors)
      DN_CUDA(cudaMemcpyAsync(colors, p->out_colors.p, 3 * n, cudaMemcpyDeviceToHost, p->stream));
    if (labels)
      DN_CUDA(cudaMemcpyAsync(labels, p->out_labels.p, n, cudaMemcpyDeviceToHost, p->stream));
  }
  DN_CUDA(cudaStreamSynchronize(p->stream));
  return DN_OK;
}

// ----------------------------------------------------------------- batch
dn_status dn_batch_create(dn_batch** out) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(out, "NULL output");
  *out = nullptr;
  DN_TRY(need_device());
  auto b = std::make_unique<dn_batch>();
  DN_TRY(b->eng.init());
  *out = b.release();
  return DN_OK;
}
dn_status dn_batch_destroy(dn_batch* b) {
  const dn::DeviceRestore device_restore_;
  delete b;
  return DN_OK;
}
dn_status dn_batch_add_view(dn_batch* b, const double* K, const double* R, const double* t,
                            const uint8_t* image, const uint8_t* mask, int width, int height,
                            int stride, int* view_id) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  return b->eng.add_view(K, R, t, image, mask, width, height, stride, view_id);
}
dn_status dn_batch_add_depthmap(dn_batch* b, int ref_view, const int* matching, int n,
                                double min_depth, double max_depth, int* map_id) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  DN_CHECK(matching || n == 0, "NULL matching view list");
  for (int k = 0; k < n; ++k) DN_CHECK(matching[k] != ref_view, "a view cannot match itself");
  return b->eng.add_map(ref_view, matching, n, min_depth, max_depth, map_id);
}
dn_status dn_batch_set_clean_views(dn_batch* b, int map_id, const int* other_maps, int n) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  DN_CHECK(map_id >= 0 && map_id < (int)b->eng.maps.size(), "depthmap id out of range");
  DN_CHECK(n >= 0 && n <= dn::kMaxNbr, "at most 16 cleaner views");
  auto& m = *b->eng.maps[map_id];
  m.clean_maps.clear();
  for (int k = 0; k < n; ++k) {
    DN_CHECK(other_maps[k] >= 0 && other_maps[k] < (int)b->eng.maps.size() && other_maps[k] != map_id,
             "cleaner view id out of range");
    m.clean_maps.push_back(other_maps[k]);
  }
  b->eng.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_params(dn_batch* b, int patch_size, float min_patch_sd, int iterations,
                              float same_depth_threshold, int min_consistent_views,
                              uint64_t seed) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  const int hpz = (patch_size - 1) / 2;
  DN_CHECK(hpz >= 1 && hpz <= dn::kMaxHpz, "patch size must be in 3..12");
  DN_CHECK(iterations >= 0 && iterations <= 1000, "iterations must be 0..1000");
  b->eng.patch = patch_size;
  b->eng.min_var = min_patch_sd * min_patch_sd;
  b->eng.iterations = iterations;
  b->eng.same_depth_thr = same_depth_threshold;
  b->eng.min_consistent = min_consistent_views;
  b->eng.seed = seed;
  b->eng.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_schedule(dn_batch* b, int half_passes, int use_near, int use_far,
                                int n_refine, float depth_range0, float normal_range0) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  DN_CHECK(half_passes >= -1 && half_passes <= 2000, "half_passes must be -1..2000");
  DN_CHECK(n_refine >= 0 && n_refine <= 12, "n_refine must be 0..12");
  DN_CHECK(depth_range0 >= 0.f && normal_range0 >= 0.f, "ranges must be >= 0");
  Engine& e = b->eng;
  e.half_passes = half_passes;
  e.use_near = use_near ? 1 : 0;
  e.use_far = use_far ? 1 : 0;
  e.n_refine = n_refine;
  e.depth_range0 = depth_range0;
  e.normal_range0 = normal_range0;
  e.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_candidate_views(dn_batch* b, int mode) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  DN_CHECK(mode >= 0 && mode <= 2,
           "candidate view mode must be 0 (all views), 1 (sample half-passes) or 2 (sample)");
  b->eng.sample_hp = mode;
  b->eng.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_knight_moves(dn_batch* b, int on) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  b->eng.use_knight = on ? 1 : 0;
  b->eng.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_active_pixels(dn_batch* b, int on, float min_change) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  DN_CHECK(min_change >= 0.f && min_change < 1.f, "min_change must be in [0, 1)");
  b->eng.active = on ? 1 : 0;
  b->eng.active_tol = min_change;
  b->eng.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_init_fallback(dn_batch* b, int on) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  b->eng.init_fallback = on ? 1 : 0;
  b->eng.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_active_seed(dn_batch* b, float min_score) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  DN_CHECK(min_score >= 0.f && min_score <= 1.f, "min_score must be in [0, 1]");
  b->eng.seed_score = min_score;
  b->eng.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_active_lists(dn_batch* b, int on) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  b->eng.active_lists = on ? 1 : 0;
  b->eng.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_proposal_scale(dn_batch* b, int ref_dim) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  DN_CHECK(ref_dim >= 0, "ref_dim must be >= 0");
  b->eng.prop_ref_dim = ref_dim;
  b->eng.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_proposal_net(dn_batch* b, const uint16_t* weights, const float* biases,
                                    int n_planes, int stride) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  Engine& e = b->eng;
  DN_CUDA(cudaSetDevice(e.device));
  if (!weights) {
    e.prop_on = false;
    e.d_prop_w.release();
    e.d_prop_b.release();
    e.invalidate();
    return DN_OK;
  }
  DN_CHECK(biases, "biases must not be NULL");
  DN_CHECK(n_planes >= 1 && n_planes <= dn::kMaxSweepPlanes, "n_planes must be 1..15");
  DN_CHECK(stride == 1 || stride == 2 || stride == 4 || stride == 8, "stride must be 1, 2, 4 or 8");
  // Layers 0-4: [32][288]; layer 5: [4][288] stored in a [32][288] slot
  // whose rows 4..31 stay zero (the kernel reads only cout rows).
  constexpr int kL = Engine::kPropLayers, kRow = 9 * 32;
  std::vector<uint16_t> w((size_t)kL * 32 * kRow, 0);
  std::vector<float> bias((size_t)kL * 32, 0.f);
  size_t off = 0;
  for (int k = 0; k < kL; ++k) {
    const int cout = k == kL - 1 ? 4 : 32;
    std::memcpy(w.data() + (size_t)k * 32 * kRow, weights + off, (size_t)cout * kRow * 2);
    std::memcpy(bias.data() + 32 * k, biases + 32 * k, (size_t)cout * sizeof(float));
    off += (size_t)cout * kRow;
  }
  for (float v : bias) DN_CHECK(std::isfinite(v), "biases must be finite");
  DN_CUDA(e.d_prop_w.alloc(w.size()));
  DN_CUDA(e.d_prop_b.alloc(bias.size()));
  DN_CUDA(cudaMemcpyAsync(e.d_prop_w.p, w.data(), w.size() * 2, cudaMemcpyHostToDevice, e.stream));
  DN_CUDA(cudaMemcpyAsync(e.d_prop_b.p, bias.data(), bias.size() * sizeof(float),
                          cudaMemcpyHostToDevice, e.stream));
  DN_CUDA(cudaStreamSynchronize(e.stream));
  e.prop_on = true;
  e.prop_planes = n_planes;
  e.prop_stride = stride;
  e.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_init(dn_batch* b, int map_id, const float* planes) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  return b->eng.set_init(map_id, planes);
}
dn_status dn_batch_run(dn_batch* b, unsigned flags) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  Engine& e = b->eng;
  DN_CUDA(cudaSetDevice(e.device));
  DN_TRY(e.check_params(Mode::kPatchMatch));
  DN_TRY(e.prepare());
  DN_CHECK(!(flags & DN_RUN_PRUNE) || (flags & DN_RUN_CLEAN),
           "DN_RUN_PRUNE prunes the cleaned depthmaps: add DN_RUN_CLEAN");
  const bool use_graph = (flags & DN_RUN_GRAPH) != 0;
  const bool timing = (flags & DN_RUN_TIMING) != 0;
  const bool learned = (flags & DN_RUN_LEARNED) != 0;
  DN_CHECK(!learned || (e.prop_on && e.d_prop_w.p),
           "DN_RUN_LEARNED needs a network (dn_batch_set_proposal_net)");
  e.timed = timing;
  if (!(flags & DN_RUN_CLEAN) && timing) {
    // No cleaner stage: its event marks the end of the run.
  }
  if (use_graph && e.graph && e.graph_flags == flags) {
    DN_CUDA(cudaGraphLaunch(e.graph, e.stream));
    b->ran = true;
    e.computed = true;
    return DN_OK;
  }
  if (use_graph) {
    if (e.graph) {
      cudaGraphExecDestroy(e.graph);
      e.graph = nullptr;
    }
    // Allocations and host-to-device table uploads happen before capture.
    if (flags & DN_RUN_CLEAN) DN_TRY(e.prepare_clean());
    if (flags & DN_RUN_PRUNE) DN_TRY(e.prepare_prune());
    cudaGraph_t g = nullptr;
    DN_CUDA(cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeThreadLocal));
    dn_status s = e.enqueue(Mode::kPatchMatch, timing, learned, (flags & DN_RUN_CLEAN) != 0,
                            (flags & DN_RUN_PRUNE) != 0);
    if (s == DN_OK && (flags & DN_RUN_CLEAN) && !e.tail_done) s = e.enqueue_clean(timing);
    if (s == DN_OK && (flags & DN_RUN_PRUNE) && !e.tail_done) s = e.enqueue_prune();
    cudaError_t ce = cudaStreamEndCapture(e.stream, &g);
    if (s != DN_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    DN_CUDA(ce);
    cudaError_t ie = cudaGraphInstantiate(&e.graph, g, 0);
    cudaGraphDestroy(g);
    DN_CUDA(ie);
    e.graph_flags = flags;
    DN_CUDA(cudaGraphLaunch(e.graph, e.stream));
  } else {
    if (flags & DN_RUN_CLEAN) DN_TRY(e.prepare_clean());
    if (flags & DN_RUN_PRUNE) DN_TRY(e.prepare_prune());
    DN_TRY(e.enqueue(Mode::kPatchMatch, timing, learned, (flags & DN_RUN_CLEAN) != 0,
                     (flags & DN_RUN_PRUNE) != 0));
    if ((flags & DN_RUN_CLEAN) && !e.tail_done) DN_TRY(e.enqueue_clean(timing));
    if ((flags & DN_RUN_PRUNE) && !e.tail_done) DN_TRY(e.enqueue_prune());
  }
  b->ran = true;
  e.computed = true;
  return DN_OK;
}
dn_status dn_batch_synchronize(dn_batch* b) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  DN_CUDA(cudaSetDevice(b->eng.device));
  return b->eng.finish();
}
dn_status dn_batch_get_depthmap(dn_batch* b, int map_id, float* depth, float* plane,
                                float* score, int32_t* nghbr, float* clean) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  return b->eng.fetch(map_id, depth, plane, score, nghbr, clean);
}
dn_status dn_batch_get_depths(dn_batch* b, int n, const int* map_ids, float* const* depths,
                              int clean) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  return b->eng.fetch_depths(n, map_ids, depths, clean);
}
dn_status dn_batch_get_depths_async(dn_batch* b, int n, const int* map_ids, float* const* depths,
                                    int clean) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  return b->eng.fetch_depths_async(n, map_ids, depths, clean);
}
dn_status dn_batch_upload_view_image(dn_batch* b, int view_id, const uint8_t* image, int stride) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  return b->eng.upload_view_image(view_id, image, stride);
}
dn_status dn_batch_pruned_count(dn_batch* b, int64_t* count) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b && count, "NULL argument");
  Engine& e = b->eng;
  DN_CHECK(e.d_prune_counts.p, "no pruner run yet (DN_RUN_PRUNE)");
  DN_CUDA(cudaSetDevice(e.device));
  std::vector<unsigned long long> c(e.maps.size());
  DN_CUDA(cudaMemcpy(c.data(), e.d_prune_counts.p, c.size() * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost));
  int64_t t = 0;
  for (auto v : c) t += (int64_t)v;
  *count = t;
  return DN_OK;
}
dn_status dn_batch_get_points(dn_batch* b, int map_id, float* points, float* normals,
                              uint8_t* colors, uint8_t* labels, int64_t capacity, int64_t* count) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b && count, "NULL argument");
  Engine& e = b->eng;
  DN_CHECK(map_id >= 0 && map_id < (int)e.maps.size(), "depthmap id out of range");
  DN_CHECK(e.d_prune_counts.p, "no pruner run yet (DN_RUN_PRUNE)");
  DN_CUDA(cudaSetDevice(e.device));
  unsigned long long c = 0;
  DN_CUDA(cudaMemcpy(&c, e.d_prune_counts.p + map_id, sizeof(c), cudaMemcpyDeviceToHost));
  *count = (int64_t)c;
  if (!points && !normals && !colors && !labels) return DN_OK;
  DN_CHECK(capacity >= (int64_t)c, "capacity is smaller than the pruned point count");
  const Map& m = *e.maps[map_id];
  const size_t n = (size_t)c;
  if (n) {
    if (points) DN_CUDA(cudaMemcpy(points, m.prune_points.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost));
    if (normals) DN_CUDA(cudaMemcpy(normals, m.prune_normals.p, 3 * n * sizeof(float), cudaMemcpyDeviceToHost));
    if (colors) DN_CUDA(cudaMemcpy(colors, m.prune_colors.p, 3 * n, cudaMemcpyDeviceToHost));
    if (labels) DN_CUDA(cudaMemcpy(labels, m.prune_labels.p, n, cudaMemcpyDeviceToHost));
  }
  return DN_OK;
}
dn_status dn_batch_last_taps(dn_batch* b, uint64_t* taps) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  return b->eng.taps(taps);
}
dn_status dn_batch_set_view_image(dn_batch* b, int view_id, const uint8_t* image, int stride) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  return b->eng.set_view_image(view_id, image, stride);
}
dn_status dn_batch_last_timings(dn_batch* b, float* out, int n, uint64_t* taps_out) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  return b->eng.timings(out, n, taps_out);
}
static dn_status set_tuning(Engine& e, int bx, int by, int variant) {
  DN_CHECK(bx >= 32 && bx % 32 == 0 && by >= 1 && bx * by <= 128,
           "block shape must have bx a multiple of 32 and bx * by <= 128");
  // variant = lanes per pixel (1, 2, 4, 8) + 16 for the persistent launch.
  DN_CHECK(variant >= 0 && variant < 32, "variant must be lanes (1, 2, 4, 8) + 16 (persistent)");
  const int lanes = variant & 15;
  DN_CHECK(lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8,
           "lanes per pixel must be 1, 2, 4 or 8");
  DN_CHECK(!(variant & 16) || (bx == 32 && by == 4),
           "the persistent launch uses 32 x 4 thread blocks");
  e.bx = bx;
  e.by = by;
  e.variant = lanes;
  e.persistent = (variant & 16) ? 1 : 0;
  e.invalidate();
  return DN_OK;
}
dn_status dn_batch_set_tuning(dn_batch* b, int bx, int by, int variant) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  return set_tuning(b->eng, bx, by, variant);
}
dn_status dn_estimator_set_tuning(dn_estimator* est, int bx, int by, int variant) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(est, "NULL estimator");
  return set_tuning(est->eng, bx, by, variant);
}
dn_status dn_batch_timer_record(dn_batch* b, int slot) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  DN_CHECK(slot == 0 || slot == 1, "timer slot must be 0 or 1");
  DN_CUDA(cudaSetDevice(b->eng.device));
  // The timer covers the pipelined host copies too: the batch stream first
  // waits for everything enqueued on the I/O streams.
  DN_TRY(b->eng.join_io());
  DN_CUDA(cudaEventRecord(b->eng.ev[5 + slot], b->eng.stream));
  return DN_OK;
}
dn_status dn_batch_timer_elapsed(dn_batch* b, float* ms) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b && ms, "NULL argument");
  DN_CUDA(cudaSetDevice(b->eng.device));
  DN_CUDA(cudaEventSynchronize(b->eng.ev[6]));
  DN_CUDA(cudaEventElapsedTime(ms, b->eng.ev[5], b->eng.ev[6]));
  return DN_OK;
}
dn_status dn_batch_copy_depth_device(dn_batch* b, int map_id, float* d_out) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b, "NULL batch");
  DN_CHECK(d_out, "NULL output");
  Engine& e = b->eng;
  DN_CHECK(map_id >= 0 && map_id < (int)e.maps.size(), "depthmap id out of range");
  DN_CUDA(cudaSetDevice(e.device));
  const Map& m = *e.maps[map_id];
  const View& r = *e.views[m.ref];
  DN_CUDA(cudaMemcpyAsync(d_out, m.depth.p, (size_t)r.W * r.H * sizeof(float),
                          cudaMemcpyDeviceToDevice, e.stream));
  return DN_OK;
}

dn_status dn_batch_sweep_features(dn_batch* b, void* feat, int64_t map_stride, int n_planes,
                                  int stride) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b && feat, "NULL argument");
  DN_CHECK(n_planes >= 1 && n_planes <= dn::kMaxSweepPlanes, "n_planes must be 1..15");
  DN_CHECK(stride == 1 || stride == 2 || stride == 4 || stride == 8, "stride must be 1, 2, 4 or 8");
  Engine& e = b->eng;
  DN_CUDA(cudaSetDevice(e.device));
  DN_CHECK(e.patch == 7, "the learned initialisation uses the 7 x 7 patch");
  for (auto& m : e.maps) {
    const View& r = *e.views[m->ref];
    const int64_t grid = (int64_t)((r.W + stride - 1) / stride) * ((r.H + stride - 1) / stride);
    DN_CHECK(grid * dn::kFeatC <= map_stride, "map_stride too small");
  }
  DN_TRY(e.check_params(Mode::kPatchMatch));
  DN_TRY(e.prepare());
  // Tiles of (bx / lanes) x by grid points, uploaded before the launch.
  const int lanes = e.variant, pxs = e.bx / lanes;
  std::vector<int4> tl;
  for (size_t k = 0; k < e.maps.size(); ++k) {
    const View& r = *e.views[e.maps[k]->ref];
    const int Ws = (r.W + stride - 1) / stride, Hs = (r.H + stride - 1) / stride;
    for (int y = 0; y < (Hs + e.by - 1) / e.by; ++y)
      for (int x = 0; x < (Ws + pxs - 1) / pxs; ++x) tl.push_back(make_int4((int)k, x, y, 0));
  }
  DN_CUDA(e.d_tiles_sweep.alloc(std::max<size_t>(tl.size(), 1)));
  DN_CUDA(cudaMemcpyAsync(e.d_tiles_sweep.p, tl.data(), tl.size() * sizeof(int4),
                          cudaMemcpyHostToDevice, e.stream));
  DN_CUDA(cudaStreamSynchronize(e.stream));
  dn::LaunchArgs a = e.args(false);
  a.tiles = e.d_tiles_sweep.p;
  a.n_tiles = (int)tl.size();
  DN_CUDA(dn::launch_sweep(a, static_cast<__nv_bfloat16*>(feat), map_stride, n_planes, stride,
                           e.stream));
  return DN_OK;
}
dn_status dn_batch_targets(dn_batch* b, float* target, int64_t map_stride, float min_score,
                           int stride) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b && target, "NULL argument");
  DN_CHECK(stride == 1 || stride == 2 || stride == 4 || stride == 8, "stride must be 1, 2, 4 or 8");
  Engine& e = b->eng;
  DN_CHECK(e.computed, "no PatchMatch result computed yet");
  DN_CUDA(cudaSetDevice(e.device));
  for (size_t k = 0; k < e.maps.size(); ++k) {
    const Map& m = *e.maps[k];
    const View& r = *e.views[m.ref];
    const int64_t grid = (int64_t)((r.W + stride - 1) / stride) * ((r.H + stride - 1) / stride);
    DN_CHECK(grid * 4 <= map_stride, "map_stride too small");
    DN_CUDA(dn::launch_planes_to_target(m.state.p, m.score.p, r.W, r.H, stride, e.d_maps.p,
                                        (int)k, min_score, target + k * map_stride, e.stream));
  }
  return DN_OK;
}
dn_status dn_batch_init_from_output(dn_batch* b, int map_id, const float* out) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(b && out, "NULL argument");
  Engine& e = b->eng;
  DN_CHECK(map_id >= 0 && map_id < (int)e.maps.size(), "depthmap id out of range");
  DN_CUDA(cudaSetDevice(e.device));
  Map& m = *e.maps[map_id];
  const View& r = *e.views[m.ref];
  const size_t npx = (size_t)r.W * r.H;
  if (!m.has_init) {
    DN_CUDA(m.init.alloc(3 * npx));
    m.has_init = true;
    e.invalidate();
  }
  DN_TRY(e.prepare());
  DN_CUDA(dn::launch_output_to_planes(out, r.W, r.H, e.d_maps.p, map_id, m.init.p, e.stream));
  return DN_OK;
}

static bool nn_shape_ok(int cin, int cout) { return cin == 32 && (cout == 32 || cout == 4); }

static dn_status nn_forward(cudaError_t (*fn)(const dn::ConvArgs&, cudaStream_t), const void* x,
                            const void* w, const float* bias, int64_t n_pix, int H, int W, int cin,
                            int cout, int relu, void* y, float* y32, void* stream) {
  DN_CHECK(x && w && bias && (y || y32), "NULL argument");
  DN_CHECK(nn_shape_ok(cin, cout), "supported shapes: cin 32, cout 32 or 4");
  DN_CHECK(H > 0 && W > 0 && n_pix > 0 && n_pix % ((int64_t)H * W) == 0, "bad n_pix / H / W");
  dn::ConvArgs c{};
  c.x = static_cast<const __nv_bfloat16*>(x);
  c.w = static_cast<const __nv_bfloat16*>(w);
  c.bias = bias;
  c.n_pix = n_pix;
  c.H = H;
  c.W = W;
  c.cin = cin;
  c.cout = cout;
  c.relu = relu;
  c.y = static_cast<__nv_bfloat16*>(y);
  c.y32 = y32;
  DN_CUDA(fn(c, static_cast<cudaStream_t>(stream)));
  return DN_OK;
}
dn_status dn_nn_conv3x3_forward(const void* x, const void* w, const float* bias, int64_t n_pix,
                                int H, int W, int cin, int cout, int relu, void* y, float* y32,
                                void* stream) {
  const dn::DeviceRestore device_restore_;
  return nn_forward(dn::conv3x3_forward, x, w, bias, n_pix, H, W, cin, cout, relu, y, y32, stream);
}
dn_status dn_nn_conv3x3_forward_mma_sync(const void* x, const void* w, const float* bias,
                                         int64_t n_pix, int H, int W, int cin, int cout, int relu,
                                         void* y, float* y32, void* stream) {
  const dn::DeviceRestore device_restore_;
  return nn_forward(dn::conv3x3_forward_mma_sync, x, w, bias, n_pix, H, W, cin, cout, relu, y, y32,
                    stream);
}
dn_status dn_nn_synchronize(void* stream) {
  const dn::DeviceRestore device_restore_;
  DN_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  const int e = dn::take_tc_error();
  DN_CHECK(e >= 0, "could not read the tensor-core error word");
  if (e) {
    g_last_error = "a tensor-core convolution's bounded wait expired";
    return DN_TIMEOUT;
  }
  return DN_OK;
}
dn_status dn_nn_conv3x3_backward(const void* dy, const void* x, const void* w,
                                 const void* x_mask, int64_t n_pix, int H, int W, int cin,
                                 int cout, void* dx, float* dw, float* db, void* wt_scratch,
                                 void* stream) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(dy && x && w && dw && db && wt_scratch, "NULL argument");
  DN_CHECK(nn_shape_ok(cin, cout), "supported shapes: cin 32, cout 32 or 4");
  DN_CHECK(H > 0 && W > 0 && n_pix > 0 && n_pix % ((int64_t)H * W) == 0, "bad n_pix / H / W");
  dn::ConvArgs c{};
  c.x = static_cast<const __nv_bfloat16*>(x);
  c.w = static_cast<const __nv_bfloat16*>(w);
  c.n_pix = n_pix;
  c.H = H;
  c.W = W;
  c.cin = cin;
  c.cout = cout;
  c.dy = static_cast<const __nv_bfloat16*>(dy);
  c.x_mask = static_cast<const __nv_bfloat16*>(x_mask);
  c.dx = static_cast<__nv_bfloat16*>(dx);
  c.dw = dw;
  c.db = db;
  DN_CUDA(dn::conv3x3_backward(c, static_cast<__nv_bfloat16*>(wt_scratch),
                               static_cast<cudaStream_t>(stream)));
  return DN_OK;
}
int64_t dn_nn_backward_scratch_bytes(int64_t n_pix, int cout) {
  // Flipped weights (32 x 288 BF16), then the gradient padded to 32 channels.
  const int64_t w = (int64_t)32 * 288 * 2;
  return cout == 32 ? w : w + n_pix * 32 * 2;
}
dn_status dn_nn_conv3x3_backward_tc(const void* dy, const void* x, const void* w,
                                    const void* x_mask, int64_t n_pix, int H, int W, int cin,
                                    int cout, void* dx, float* dw, float* db, void* scratch,
                                    int64_t scratch_bytes, void* stream) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(dy && x && w && dw && db && scratch, "NULL argument");
  DN_CHECK(nn_shape_ok(cin, cout), "supported shapes: cin 32, cout 32 or 4");
  DN_CHECK(H > 0 && W > 0 && n_pix > 0 && n_pix % ((int64_t)H * W) == 0, "bad n_pix / H / W");
  DN_CHECK(!dx || scratch_bytes >= dn_nn_backward_scratch_bytes(n_pix, cout),
           "scratch smaller than dn_nn_backward_scratch_bytes");
  dn::ConvArgs c{};
  c.x = static_cast<const __nv_bfloat16*>(x);
  c.w = static_cast<const __nv_bfloat16*>(w);
  c.n_pix = n_pix;
  c.H = H;
  c.W = W;
  c.cin = cin;
  c.cout = cout;
  c.dy = static_cast<const __nv_bfloat16*>(dy);
  c.x_mask = static_cast<const __nv_bfloat16*>(x_mask);
  c.dx = static_cast<__nv_bfloat16*>(dx);
  c.dw = dw;
  c.db = db;
  __nv_bfloat16* wt = static_cast<__nv_bfloat16*>(scratch);
  DN_CUDA(dn::conv3x3_backward_tc(c, wt, wt + 32 * 288, static_cast<cudaStream_t>(stream)));
  return DN_OK;
}
dn_status dn_nn_l1_loss(const float* pred, const float* target, int64_t n_pix,
                        float normal_weight, void* dpred, float* loss_sum, float* count,
                        void* stream) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(pred && target && dpred && loss_sum && count && n_pix > 0, "bad argument");
  DN_CUDA(dn::launch_l1_loss(pred, target, n_pix, normal_weight,
                             static_cast<__nv_bfloat16*>(dpred), loss_sum, count,
                             static_cast<cudaStream_t>(stream)));
  return DN_OK;
}
dn_status dn_nn_adam(float* w, float* m, float* v, const float* grad, int n, const float* count,
                     float lr, float beta1, float beta2, float eps, float bc1, float bc2,
                     void* w16, void* stream) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(w && m && v && grad && count && n > 0, "bad argument");
  DN_CUDA(dn::launch_adam(w, m, v, grad, n, count, lr, beta1, beta2, eps, bc1, bc2,
                          static_cast<__nv_bfloat16*>(w16), static_cast<cudaStream_t>(stream)));
  return DN_OK;
}

dn_status dn_postprocess_depth(const float* depth, float* out, int width, int height) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(depth && out, "NULL buffer");
  DN_CHECK(width >= 1 && height >= 1 && width <= 16384 && height <= 16384, "bad size");
  DN_TRY(need_device());
  const size_t n = (size_t)width * height;
  DevBuf<float> a, b;
  DN_CUDA(a.alloc(n));
  DN_CUDA(b.alloc(n));
  DN_CUDA(cudaMemcpy(a.p, depth, n * sizeof(float), cudaMemcpyHostToDevice));
  DN_CUDA(dn::launch_postprocess_plain(a.p, b.p, width, height, 0));
  DN_CUDA(cudaMemcpy(out, b.p, n * sizeof(float), cudaMemcpyDeviceToHost));
  return DN_OK;
}

dn_status dn_check_bounded_wait(int blocks, int64_t max_spins, float* ms) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(blocks >= 1 && blocks <= 64, "blocks must be 1..64");
  DN_CHECK(max_spins >= 1 && max_spins <= (int64_t)1 << 24, "max_spins must be 1..2^24");
  DN_TRY(need_device());
  DevBuf<unsigned> sync;
  DevBuf<int> err;
  DN_CUDA(sync.alloc(2));
  DN_CUDA(err.alloc(1));
  DN_CUDA(cudaMemset(sync.p, 0, 2 * sizeof(unsigned)));
  DN_CUDA(cudaMemset(err.p, 0, sizeof(int)));
  cudaEvent_t e0, e1;
  DN_CUDA(cudaEventCreate(&e0));
  DN_CUDA(cudaEventCreate(&e1));
  DN_CUDA(cudaEventRecord(e0, 0));
  const cudaError_t le = dn::launch_barrier_expiry(sync.p, err.p, blocks, max_spins, 0);
  DN_CUDA(cudaEventRecord(e1, 0));
  const cudaError_t se = cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  DN_CUDA(le);
  DN_CUDA(se);
  if (ms) *ms = t;
  int flag = 0;
  DN_CUDA(cudaMemcpy(&flag, err.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) return fail(DN_TIMEOUT, "a bounded device-side wait expired (as this check intends)");
  return fail(DN_DEVICE_ERROR, "the never-opening barrier did not report its expiry");
}

dn_status dn_fp32_peak(double* tflops, double* ms) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(tflops && ms, "NULL output");
  DN_TRY(need_device());
  DN_CUDA(dn::fp32_peak(tflops, ms));
  return DN_OK;
}
dn_status dn_walk_ceiling(double* gtaps, double* ms) {
  const dn::DeviceRestore device_restore_;
  DN_CHECK(gtaps && ms, "NULL output");
  DN_TRY(need_device());
  DN_CUDA(dn::walk_ceiling(gtaps, ms));
  return DN_OK;
}

}  // extern "C"
