// C entry points over the reference's legacy dense classes
// (opensfm/src/lib/dense/depthmap.h:57-153), so tests and the CPU baseline can
// drive the compiled reference through ctypes.  TEST INFRASTRUCTURE ONLY:
// built by oracle/Makefile into oracle/_ref/, never linked by the product.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "depthmap.h"

using dense::DepthmapCleaner;
using dense::DepthmapEstimator;
using dense::DepthmapEstimatorResult;
using dense::DepthmapPruner;

namespace {
struct EstimatorBox {
  DepthmapEstimator est;
  int width = 0, height = 0, patch_size = 7;
};
struct PrunerBox {
  DepthmapPruner pruner;
  std::vector<float> points, normals;
  std::vector<unsigned char> colors, labels;
};
void copy_result(const DepthmapEstimatorResult& r, float* depth, float* plane,
                 float* score, int32_t* nghbr) {
  const size_t n = size_t(r.depth.rows) * r.depth.cols;
  std::memcpy(depth, r.depth.data(), n * sizeof(float));
  std::memcpy(plane, r.plane.data(), n * 3 * sizeof(float));
  std::memcpy(score, r.score.data(), n * sizeof(float));
  std::memcpy(nghbr, r.nghbr.data(), n * sizeof(int32_t));
}
}  // namespace

extern "C" {

void ref_srand(unsigned seed) { std::srand(seed); }

void* ref_est_new() { return new EstimatorBox(); }
void ref_est_free(void* h) { delete static_cast<EstimatorBox*>(h); }
void ref_est_add_view(void* h, const double* K, const double* R, const double* t,
                      const uint8_t* image, const uint8_t* mask, int width, int height) {
  auto* b = static_cast<EstimatorBox*>(h);
  if (b->width == 0) {
    b->width = width;
    b->height = height;
  }
  b->est.AddView(K, R, t, image, mask, width, height);
}
void ref_est_set_depth_range(void* h, double mn, double mx, int n) {
  static_cast<EstimatorBox*>(h)->est.SetDepthRange(mn, mx, n);
}
void ref_est_set_patchmatch_iterations(void* h, int n) {
  static_cast<EstimatorBox*>(h)->est.SetPatchMatchIterations(n);
}
void ref_est_set_patch_size(void* h, int n) {
  auto* b = static_cast<EstimatorBox*>(h);
  b->patch_size = n;
  b->est.SetPatchSize(n);
}
void ref_est_set_min_patch_sd(void* h, float sd) {
  static_cast<EstimatorBox*>(h)->est.SetMinPatchSD(sd);
}
// mode 0: ComputeBruteForce, 1: ComputePatchMatch, 2: ComputePatchMatchSample
void ref_est_compute(void* h, int mode, float* depth, float* plane, float* score,
                     int32_t* nghbr) {
  auto* b = static_cast<EstimatorBox*>(h);
  DepthmapEstimatorResult r;
  if (mode == 0) b->est.ComputeBruteForce(&r);
  else if (mode == 1) b->est.ComputePatchMatch(&r);
  else b->est.ComputePatchMatchSample(&r);
  copy_result(r, depth, plane, score, nghbr);
}
// ComputePlaneScore (depthmap.cc:408-419) for every interior pixel with the
// given per-pixel planes (H x W x 3); border pixels get score 0, nghbr 0.
void ref_est_score_planes(void* h, const float* planes, float* score, int32_t* nghbr) {
  auto* b = static_cast<EstimatorBox*>(h);
  const int W = b->width, H = b->height, hpz = (b->patch_size - 1) / 2;
  for (int i = 0; i < H; ++i)
    for (int j = 0; j < W; ++j) {
      const size_t p = size_t(i) * W + j;
      score[p] = 0.0f;
      nghbr[p] = 0;
      if (i < hpz || i >= H - hpz || j < hpz || j >= W - hpz) continue;
      cv::Vec3f plane(planes[3 * p], planes[3 * p + 1], planes[3 * p + 2]);
      float s;
      int n;
      b->est.ComputePlaneScore(i, j, plane, &s, &n);
      score[p] = s;
      nghbr[p] = n;
    }
}
float ref_est_plane_image_score(void* h, int i, int j, const float* plane, int other) {
  cv::Vec3f v(plane[0], plane[1], plane[2]);
  return static_cast<EstimatorBox*>(h)->est.ComputePlaneImageScore(i, j, v, other);
}
float ref_patch_variance(void* h, int i, int j) {
  return static_cast<EstimatorBox*>(h)->est.PatchVariance(i, j);
}
void ref_median5(const float* src, float* dst, int width, int height) {
  cv::Mat s(height, width, CV_32F, (void*)src), d;
  cv::medianBlur(s, d, 5);
  std::memcpy(dst, d.data(), size_t(width) * height * sizeof(float));
}
void ref_inv3(const double* a, double* out) {
  cv::Matx33d m(a);
  cv::Matx33d r = m.inv();
  std::memcpy(out, r.val, 9 * sizeof(double));
}

void* ref_cleaner_new() { return new DepthmapCleaner(); }
void ref_cleaner_free(void* h) { delete static_cast<DepthmapCleaner*>(h); }
void ref_cleaner_set_same_depth_threshold(void* h, float t) {
  static_cast<DepthmapCleaner*>(h)->SetSameDepthThreshold(t);
}
void ref_cleaner_set_min_consistent_views(void* h, int n) {
  static_cast<DepthmapCleaner*>(h)->SetMinConsistentViews(n);
}
void ref_cleaner_add_view(void* h, const double* K, const double* R, const double* t,
                          const float* depth, int width, int height) {
  static_cast<DepthmapCleaner*>(h)->AddView(K, R, t, depth, width, height);
}
void ref_cleaner_clean(void* h, float* out, int width, int height) {
  cv::Mat m;
  static_cast<DepthmapCleaner*>(h)->Clean(&m);
  std::memcpy(out, m.data(), size_t(width) * height * sizeof(float));
}

void* ref_pruner_new() { return new PrunerBox(); }
void ref_pruner_free(void* h) { delete static_cast<PrunerBox*>(h); }
void ref_pruner_set_same_depth_threshold(void* h, float t) {
  static_cast<PrunerBox*>(h)->pruner.SetSameDepthThreshold(t);
}
void ref_pruner_add_view(void* h, const double* K, const double* R, const double* t,
                         const float* depth, const float* plane, const uint8_t* color,
                         const uint8_t* label, int width, int height) {
  static_cast<PrunerBox*>(h)->pruner.AddView(K, R, t, depth, plane, color, label, width,
                                             height);
}
// Runs Prune and keeps the result; returns the number of kept points.
long ref_pruner_prune(void* h) {
  auto* b = static_cast<PrunerBox*>(h);
  b->points.clear();
  b->normals.clear();
  b->colors.clear();
  b->labels.clear();
  b->pruner.Prune(&b->points, &b->normals, &b->colors, &b->labels);
  return long(b->labels.size());
}
void ref_pruner_fetch(void* h, float* points, float* normals, uint8_t* colors,
                      uint8_t* labels) {
  auto* b = static_cast<PrunerBox*>(h);
  std::memcpy(points, b->points.data(), b->points.size() * sizeof(float));
  std::memcpy(normals, b->normals.data(), b->normals.size() * sizeof(float));
  std::memcpy(colors, b->colors.data(), b->colors.size());
  std::memcpy(labels, b->labels.data(), b->labels.size());
}

}  // extern "C"
