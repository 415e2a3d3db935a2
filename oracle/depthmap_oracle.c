/* CPU restatement of the reference's legacy dense depthmap path
 * (opensfm/src/lib/dense/src/depthmap.cc), in plain C.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load this library, and only as a
 * checker or as the timed CPU baseline; the product never links it.
 *
 * Arithmetic follows the reference step by step (float where it uses float,
 * double where it uses double, same operation order, no FP contraction:
 * build with -ffp-contract=off), so brute force, plane scoring, the cleaner,
 * the pruner and the median post-process agree bit for bit with the
 * reference compiled from its own source (checked by tests/test_oracle.py
 * against tests/golden/ and oracle/_ref/).  PatchMatch follows the
 * reference's raster schedule but draws its random numbers from a seeded
 * SplitMix64 stream instead of rand()/std::mt19937, so it is reproducible.
 *
 * Layouts: views share one size W x H; images/masks u8 [n][H][W]; K, R
 * row-major 3x3 double [n][9]; t [n][3]; depth f32 [H][W]; plane f32
 * [H][W][3]; score f32 [H][W]; nghbr i32 [H][W].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- 3x3 algebra
 * Products accumulate from +0 in index order, as cv::Matx does. */
static void m3_mul(const double* a, const double* b, double* c) {
  double r[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
      for (int k = 0; k < 3; ++k) s += a[3 * i + k] * b[3 * k + j];
      r[3 * i + j] = s;
    }
  memcpy(c, r, sizeof(r));
}
static void m3_vec(const double* a, const double* x, double* y) {
  double r[3];
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s += a[3 * i + k] * x[k];
    r[i] = s;
  }
  memcpy(y, r, sizeof(r));
}
static void m3_t(const double* a, double* b) {
  double r[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[3 * j + i] = a[3 * i + j];
  memcpy(b, r, sizeof(r));
}
/* Cofactor inverse scaled by 1/det (cv::Matx<double,3,3>::inv). */
void or_inv3(const double* a, double* r) {
#define A(i, j) a[3 * (i) + (j)]
  double d = A(0, 0) * (A(1, 1) * A(2, 2) - A(2, 1) * A(1, 2)) -
             A(0, 1) * (A(1, 0) * A(2, 2) - A(2, 0) * A(1, 2)) +
             A(0, 2) * (A(1, 0) * A(2, 1) - A(2, 0) * A(1, 1));
  if (d == 0) {
    memset(r, 0, 9 * sizeof(double));
    return;
  }
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
#undef A
}

/* ------------------------------------------------------------ per-view setup
 * depthmap.cc:146-162: Kinv_i = K_i^-1, Q_i = R_i R_0^T, a_i = Q_i t_0 - t_i. */
typedef struct {
  int n, W, H;
  const double *K, *R, *t;
  double (*Kinv)[9], (*Q)[9], (*a)[3];
  const uint8_t* img;
  const uint8_t* mask;
  int hpz;
} views_t;

static void views_init(views_t* v, int n, const double* K, const double* R, const double* t,
                       const uint8_t* img, const uint8_t* mask, int W, int H, int patch) {
  v->n = n;
  v->W = W;
  v->H = H;
  v->K = K;
  v->R = R;
  v->t = t;
  v->img = img;
  v->mask = mask;
  v->hpz = (patch - 1) / 2;
  v->Kinv = malloc(sizeof(double[9]) * (n ? n : 1));
  v->Q = malloc(sizeof(double[9]) * (n ? n : 1));
  v->a = malloc(sizeof(double[3]) * (n ? n : 1));
  double R0t[9];
  m3_t(R, R0t);
  for (int i = 0; i < n; ++i) {
    or_inv3(K + 9 * i, v->Kinv[i]);
    m3_mul(R + 9 * i, R0t, v->Q[i]);
    double qt[3];
    m3_vec(v->Q[i], t, qt);
    for (int k = 0; k < 3; ++k) v->a[i][k] = qt[k] - t[3 * i + k];
  }
}
static void views_free(views_t* v) {
  free(v->Kinv);
  free(v->Q);
  free(v->a);
}

/* ------------------------------------------------------------ plane helpers */
/* PlaneFromDepthAndNormal (depthmap.cc:120-125). */
static void plane_from_depth_normal(float x, float y, const double* Kinv, float depth,
                                    const float n[3], float out[3]) {
  double M[9], q[3] = {(double)x, (double)y, 1.0}, p[3];
  for (int k = 0; k < 9; ++k) M[k] = Kinv[k] * (double)depth;
  m3_vec(M, q, p);
  float pf[3] = {(float)p[0], (float)p[1], (float)p[2]};
  float s = 0.0f;
  for (int k = 0; k < 3; ++k) s += n[k] * pf[k];
  float denom = -s;
  float m = (1e-6f < denom) ? denom : 1e-6f;
  float inv = 1.f / m;
  for (int k = 0; k < 3; ++k) out[k] = n[k] * inv;
}

/* DepthOfPlaneBackprojection (depthmap.cc:114-118). */
static float depth_of_plane(double x, double y, const double* Kinv, const float pl[3]) {
  double r[3];
  for (int j = 0; j < 3; ++j) {
    double s = 0.0;
    for (int k = 0; k < 3; ++k) s += (double)pl[k] * Kinv[3 * k + j];
    r[j] = s;
  }
  double s = 0.0;
  s += r[0] * x;
  s += r[1] * y;
  s += r[2] * 1.0;
  float denom = (float)(-s);
  float m = (1e-6f < denom) ? denom : 1e-6f;
  return 1.0f / m;
}

/* PlaneInducedHomographyBaked (depthmap.cc:96-102): K2 (Q2 + a2 v^T) K1inv. */
static void homography(const double* K1inv, const double* Q2, const double* a2,
                       const double* K2, const float v[3], float Hf[9]) {
  double M[9], T[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double av = 0.0;
      av += a2[i] * (double)v[j];
      M[3 * i + j] = Q2[3 * i + j] + av;
    }
  m3_mul(K2, M, T);
  m3_mul(T, K1inv, T);
  for (int k = 0; k < 9; ++k) Hf[k] = (float)T[k];
}

/* LinearInterpolation (depthmap.cc:14-30): 0 outside [0, W-1) x [0, H-1). */
static float bilinear_u8(const uint8_t* im, int W, int H, float y, float x) {
  if (x < 0.0f || x >= W - 1 || y < 0.0f || y >= H - 1) return 0.0f;
  int ix = (int)x, iy = (int)y;
  float dx = x - ix, dy = y - iy;
  float i00 = im[(size_t)iy * W + ix], i01 = im[(size_t)iy * W + ix + 1];
  float i10 = im[(size_t)(iy + 1) * W + ix], i11 = im[(size_t)(iy + 1) * W + ix + 1];
  float i0 = (1 - dx) * i00 + dx * i01;
  float i1 = (1 - dx) * i10 + dx * i11;
  return (1 - dy) * i0 + dy * i1;
}
static float bilinear_f32(const float* im, int W, int H, float y, float x) {
  if (x < 0.0f || x >= W - 1 || y < 0.0f || y >= H - 1) return 0.0f;
  int ix = (int)x, iy = (int)y;
  float dx = x - ix, dy = y - iy;
  float i00 = im[(size_t)iy * W + ix], i01 = im[(size_t)iy * W + ix + 1];
  float i10 = im[(size_t)(iy + 1) * W + ix], i11 = im[(size_t)(iy + 1) * W + ix + 1];
  float i0 = (1 - dx) * i00 + dx * i01;
  float i1 = (1 - dx) * i10 + dx * i11;
  return (1 - dy) * i0 + dy * i1;
}

/* BilateralWeight (depthmap.cc:480-487). */
static float bilateral_weight(float dcolor, float dx, float dy) {
  const float dcolor_sigma = 50.0f, dx_sigma = 5.0f;
  const float dcolor_factor = 1.0f / (2 * dcolor_sigma * dcolor_sigma);
  const float dx_factor = 1.0f / (2 * dx_sigma * dx_sigma);
  return expf(-dcolor * dcolor * dcolor_factor - (dx * dx + dy * dy) * dx_factor);
}

/* ComputePlaneImageScore (depthmap.cc:441-478) with NCCEstimator
 * (depthmap.cc:46-74): local affine warp of the plane-induced homography,
 * bilateral-weighted raw-moment NCC in float. */
float or_plane_image_score_v(const views_t* V, int i, int j, const float plane[3], int other) {
  float H[9];
  homography(V->Kinv[0], V->Q[other], V->a[other], V->K + 9 * other, plane, H);
  const int hpz = V->hpz, W = V->W, Hh = V->H;
  float u = H[0] * j + H[1] * i + H[2];
  float v = H[3] * j + H[4] * i + H[5];
  float w = H[6] * j + H[7] * i + H[8];
  if (w == 0.0) return -1.0f;
  float dfdx_x = (H[0] * w - H[6] * u) / (w * w);
  float dfdx_y = (H[3] * w - H[6] * v) / (w * w);
  float dfdy_x = (H[1] * w - H[7] * u) / (w * w);
  float dfdy_y = (H[4] * w - H[7] * v) / (w * w);
  float Hx0 = u / w, Hy0 = v / w;
  const uint8_t* ref = V->img;
  const uint8_t* oth = V->img + (size_t)other * W * Hh;
  float c = ref[(size_t)i * W + j];
  float sx = 0, sy = 0, sxx = 0, syy = 0, sxy = 0, sw = 0;
  for (int dy = -hpz; dy <= hpz; ++dy)
    for (int dx = -hpz; dx <= hpz; ++dx) {
      float x1 = ref[(size_t)(i + dy) * W + j + dx];
      float x2 = Hx0 + dfdx_x * dx + dfdy_x * dy;
      float y2 = Hy0 + dfdx_y * dx + dfdy_y * dy;
      float x2v = bilinear_u8(oth, W, Hh, y2, x2);
      float wt = bilateral_weight(x1 - c, (float)dx, (float)dy);
      sx += wt * x1;
      sy += wt * x2v;
      sxx += wt * x1 * x1;
      syy += wt * x2v * x2v;
      sxy += wt * x1 * x2v;
      sw += wt;
    }
  if (sw == 0.0) return -1;
  float mx = sx / sw, my = sy / sw, mxx = sxx / sw, myy = syy / sw, mxy = sxy / sw;
  float vx = mxx - mx * mx, vy = myy - my * my;
  if (vx < 0.1 || vy < 0.1) return -1;
  return (mxy - mx * my) / sqrtf(vx * vy);
}

/* ComputePlaneScore (depthmap.cc:408-419): max over views, first max wins. */
static void plane_score(const views_t* V, int i, int j, const float plane[3], float* score,
                        int* nghbr) {
  *score = -1.0f;
  *nghbr = 0;
  for (int o = 1; o < V->n; ++o) {
    float s = or_plane_image_score_v(V, i, j, plane, o);
    if (s > *score) {
      *score = s;
      *nghbr = o;
    }
  }
}

/* --------------------------------------------------------------- RNG (port) */
typedef struct {
  uint64_t s;
} rng_t;
static uint64_t splitmix(rng_t* r) {
  uint64_t z = (r->s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static float uniform01(rng_t* r) { return (float)((splitmix(r) >> 40) * (1.0 / 16777216.0)); }
static float uniform_ab(rng_t* r, float a, float b) { return a + (b - a) * uniform01(r); }
static float normal01(rng_t* r) {
  double u1 = ((splitmix(r) >> 11) + 1.0) * (1.0 / 9007199254740993.0);
  double u2 = (splitmix(r) >> 11) * (1.0 / 9007199254740992.0);
  return (float)(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
}
static int uniform_int(rng_t* r, int a, int b) {
  return a + (int)(splitmix(r) % (uint64_t)(b - a + 1));
}

/* --------------------------------------------------------------- estimator */
typedef struct {
  float *depth, *plane, *score;
  int32_t* nghbr;
} result_t;

static void assign(result_t* R, int W, int i, int j, float d, const float pl[3], float s, int n) {
  size_t p = (size_t)i * W + j;
  R->depth[p] = d;
  R->plane[3 * p] = pl[0];
  R->plane[3 * p + 1] = pl[1];
  R->plane[3 * p + 2] = pl[2];
  R->score[p] = s;
  R->nghbr[p] = n;
}
static void check_plane(const views_t* V, result_t* R, int i, int j, const float pl[3]) {
  float s;
  int n;
  plane_score(V, i, j, pl, &s, &n);
  if (s > R->score[(size_t)i * V->W + j]) {
    float d = depth_of_plane(j, i, V->Kinv[0], pl);
    assign(R, V->W, i, j, d, pl, s, n);
  }
}
static void check_plane_image(const views_t* V, result_t* R, int i, int j, const float pl[3],
                              int o) {
  float s = or_plane_image_score_v(V, i, j, pl, o);
  if (s > R->score[(size_t)i * V->W + j]) {
    float d = depth_of_plane(j, i, V->Kinv[0], pl);
    assign(R, V->W, i, j, d, pl, s, o);
  }
}

/* Variance (depthmap.cc:32-44) of the patch around (i, j). */
static float patch_variance(const views_t* V, int i, int j) {
  const int hpz = V->hpz, n = (2 * hpz + 1) * (2 * hpz + 1);
  float buf[64 * 64];
  int c = 0;
  for (int u = -hpz; u <= hpz; ++u)
    for (int v = -hpz; v <= hpz; ++v) buf[c++] = V->img[(size_t)(i + u) * V->W + j + v];
  float sum = 0;
  for (int k = 0; k < n; ++k) sum += buf[k];
  float mean = sum / n, s2 = 0;
  for (int k = 0; k < n; ++k) s2 += (buf[k] - mean) * (buf[k] - mean);
  return s2 / n;
}
float or_patch_variance(const uint8_t* img, int W, int H, int patch, int i, int j) {
  views_t V;
  memset(&V, 0, sizeof(V));
  V.img = img;
  V.W = W;
  V.H = H;
  V.hpz = (patch - 1) / 2;
  return patch_variance(&V, i, j);
}

static void update_pixel(const views_t* V, result_t* R, int i, int j, const int adj[2][2],
                         int sample, rng_t* rng) {
  const int W = V->W;
  size_t p = (size_t)i * W + j;
  if (R->depth[p] == 0.0f) return;
  for (int k = 0; k < 2; ++k) {
    size_t q = (size_t)(i + adj[k][0]) * W + (j + adj[k][1]);
    if (R->depth[q] == 0.0f) continue;
    float pl[3] = {R->plane[3 * q], R->plane[3 * q + 1], R->plane[3 * q + 2]};
    if (sample) check_plane_image(V, R, i, j, pl, R->nghbr[q]);
    else check_plane(V, R, i, j, pl);
  }
  float depth_range = 0.02f, normal_range = 0.5f;
  int cur_n = R->nghbr[p];
  for (int k = 0; k < 6; ++k) {
    float cd = R->depth[p];
    float d = cd * expf(depth_range * normal01(rng));
    float cp[3] = {R->plane[3 * p], R->plane[3 * p + 1], R->plane[3 * p + 2]};
    if (cp[2] == 0.0) continue;
    float n[3] = {-cp[0] / cp[2] + normal_range * normal01(rng),
                  -cp[1] / cp[2] + normal_range * normal01(rng), -1.0f};
    float pl[3];
    plane_from_depth_normal((float)j, (float)i, V->Kinv[0], d, n, pl);
    if (sample) check_plane_image(V, R, i, j, pl, cur_n);
    else check_plane(V, R, i, j, pl);
    depth_range *= 0.3f;
    normal_range *= 0.8f;
  }
  if (!sample || V->n <= 2) return;
  int other = uniform_int(rng, 1, V->n - 1);
  while (other == cur_n) other = uniform_int(rng, 1, V->n - 1);
  float pl[3] = {R->plane[3 * p], R->plane[3 * p + 1], R->plane[3 * p + 2]};
  check_plane_image(V, R, i, j, pl, other);
}

void or_median5(const float* src, float* dst, int W, int H);

/* PostProcess (depthmap.cc:489-502). */
static void post_process(result_t* R, int W, int H) {
  float* m = malloc(sizeof(float) * (size_t)W * H);
  or_median5(R->depth, m, W, H);
  for (size_t p = 0; p < (size_t)W * H; ++p) {
    float d = R->depth[p];
    if (d == 0.0 || fabsf(d - m[p]) / d > 0.05) R->depth[p] = 0;
  }
  free(m);
}

/* mode 0: ComputeBruteForce (depthmap.cc:184-200); 1: ComputePatchMatch
 * (202-213); 2: ComputePatchMatchSample (215-227). */
int or_compute(int mode, int n, const double* K, const double* Rm, const double* t,
               const uint8_t* images, const uint8_t* masks, int W, int H, int patch,
               double min_depth, double max_depth, int num_planes, int iters,
               float min_patch_sd, uint64_t seed, float* depth, float* plane, float* score,
               int32_t* nghbr) {
  views_t V;
  views_init(&V, n, K, Rm, t, images, masks, W, H, patch);
  result_t R = {depth, plane, score, nghbr};
  memset(depth, 0, sizeof(float) * (size_t)W * H);
  memset(plane, 0, sizeof(float) * 3 * (size_t)W * H);
  memset(score, 0, sizeof(float) * (size_t)W * H);
  memset(nghbr, 0, sizeof(int32_t) * (size_t)W * H);
  const int hpz = V.hpz;
  if (mode == 0) {
    for (int i = hpz; i < H - hpz; ++i)
      for (int j = hpz; j < W - hpz; ++j)
        for (int d = 0; d < num_planes; ++d) {
          float dep = (float)(1 / (1 / min_depth + d * (1 / max_depth - 1 / min_depth) /
                                                      (num_planes - 1)));
          const float nrm[3] = {0, 0, -1};
          float pl[3];
          plane_from_depth_normal((float)j, (float)i, V.Kinv[0], dep, nrm, pl);
          check_plane(&V, &R, i, j, pl);
        }
    views_free(&V);
    return 0;
  }
  const int sample = (mode == 2);
  rng_t rng = {seed};
  /* RandomInitialization (237-256). */
  for (int i = hpz; i < H - hpz; ++i)
    for (int j = hpz; j < W - hpz; ++j) {
      float dep = expf(uniform_ab(&rng, (float)log(min_depth), (float)log(max_depth)));
      float nrm[3] = {uniform_ab(&rng, -1, 1), uniform_ab(&rng, -1, 1), -1};
      float pl[3];
      plane_from_depth_normal((float)j, (float)i, V.Kinv[0], dep, nrm, pl);
      int nb;
      float s;
      if (sample) {
        nb = uniform_int(&rng, n > 1 ? 1 : 0, n > 1 ? n - 1 : 0);
        s = or_plane_image_score_v(&V, i, j, pl, nb);
      } else {
        plane_score(&V, i, j, pl, &s, &nb);
      }
      assign(&R, W, i, j, dep, pl, s, nb);
    }
  /* ComputeIgnoreMask (258-269). */
  const float min_var = min_patch_sd * min_patch_sd;
  for (int i = hpz; i < H - hpz; ++i)
    for (int j = hpz; j < W - hpz; ++j) {
      int masked = masks[(size_t)i * W + j] == 0;
      int low = patch_variance(&V, i, j) < min_var;
      if (masked || low) {
        const float z[3] = {0, 0, 0};
        assign(&R, W, i, j, 0.0f, z, 0.0f, 0);
      }
    }
  const int fwd[2][2] = {{-1, 0}, {0, -1}}, bwd[2][2] = {{0, 1}, {1, 0}};
  for (int it = 0; it < iters; ++it) {
    for (int i = hpz; i < H - hpz; ++i)
      for (int j = hpz; j < W - hpz; ++j) update_pixel(&V, &R, i, j, fwd, sample, &rng);
    for (int i = H - hpz - 1; i >= hpz; --i)
      for (int j = W - hpz - 1; j >= hpz; --j) update_pixel(&V, &R, i, j, bwd, sample, &rng);
  }
  post_process(&R, W, H);
  views_free(&V);
  return 0;
}

/* The GPU's red-black schedule (kernels.cu halfpass_tile) restated with the
 * reference's arithmetic: the same RandomInitialization and
 * ComputeIgnoreMask, then `half_passes` half-passes, each updating the
 * pixels with (i + j) % 2 == colour from the other colour (which the
 * half-pass does not write, so a sequential loop equals the parallel
 * kernel).  Candidates per update, each through CheckPlaneCandidate
 * (depthmap.cc:376-385): the 4 adjacent planes, per direction the plane of
 * the best-scoring valid pixel at distances 3, 5, ..., 23, then 6
 * refinements with PatchMatchUpdatePixel's decay (depthmap.cc:334-360).
 * With `sample`, as ComputePatchMatchSample (depthmap.cc:215-227): one view
 * per candidate (CheckPlaneImageCandidate, depthmap.cc:387-396) and a
 * random other view of the current plane per update.  The
 * random numbers come from this file's generator, not the GPU's Philox
 * streams, so results agree with the GPU statistically, not bit for bit.
 * Used to show which accuracy the schedule itself reaches. */
static void redblack_check(const views_t* V, result_t* R, int i, int j, const float pl[3],
                           int sample, int view) {
  if (sample) check_plane_image(V, R, i, j, pl, view);
  else check_plane(V, R, i, j, pl);
}

static void redblack_update(const views_t* V, result_t* R, int i, int j, int sample, rng_t* rng) {
  const int W = V->W, H = V->H;
  const size_t p = (size_t)i * W + j;
  if (R->depth[p] == 0.0f) return;
  const int di[4] = {-1, 0, 1, 0}, dj[4] = {0, -1, 0, 1};
  for (int d = 0; d < 4; ++d) {
    const size_t q = (size_t)(i + di[d]) * W + (j + dj[d]);
    if (R->depth[q] == 0.0f) continue;
    const float pl[3] = {R->plane[3 * q], R->plane[3 * q + 1], R->plane[3 * q + 2]};
    redblack_check(V, R, i, j, pl, sample, R->nghbr[q]);
  }
  for (int d = 0; d < 4; ++d) {
    long best = -1;
    float best_score = -3.0f;
    for (int k = 0; k < 11; ++k) {
      const int dist = 3 + 2 * k, qi = i + di[d] * dist, qj = j + dj[d] * dist;
      if (qi < 0 || qi >= H || qj < 0 || qj >= W) break;
      const size_t q = (size_t)qi * W + qj;
      if (R->score[q] > best_score && R->depth[q] != 0.0f) {
        best_score = R->score[q];
        best = (long)q;
      }
    }
    if (best < 0) continue;
    const float pl[3] = {R->plane[3 * best], R->plane[3 * best + 1], R->plane[3 * best + 2]};
    redblack_check(V, R, i, j, pl, sample, R->nghbr[best]);
  }
  float depth_range = 0.02f, normal_range = 0.5f;
  const int cur_n = R->nghbr[p];
  for (int k = 0; k < 6; ++k) {
    const float cd = R->depth[p];
    const float d = cd * expf(depth_range * normal01(rng));
    const float cp[3] = {R->plane[3 * p], R->plane[3 * p + 1], R->plane[3 * p + 2]};
    if (cp[2] == 0.0) continue;
    float n[3] = {-cp[0] / cp[2] + normal_range * normal01(rng),
                  -cp[1] / cp[2] + normal_range * normal01(rng), -1.0f};
    float pl[3];
    plane_from_depth_normal((float)j, (float)i, V->Kinv[0], d, n, pl);
    redblack_check(V, R, i, j, pl, sample, cur_n);
    depth_range *= 0.3f;
    normal_range *= 0.8f;
  }
  if (!sample || V->n <= 2) return;
  /* A random other matching view for the current plane. */
  int other = uniform_int(rng, 1, V->n - 2);
  if (other >= R->nghbr[p]) other += 1;
  const float pl[3] = {R->plane[3 * p], R->plane[3 * p + 1], R->plane[3 * p + 2]};
  check_plane_image(V, R, i, j, pl, other);
}

int or_compute_redblack(int sample, int n, const double* K, const double* Rm, const double* t,
                        const uint8_t* images, const uint8_t* masks, int W, int H, int patch,
                        double min_depth, double max_depth, int half_passes, float min_patch_sd,
                        uint64_t seed, float* depth, float* plane, float* score, int32_t* nghbr) {
  views_t V;
  views_init(&V, n, K, Rm, t, images, masks, W, H, patch);
  result_t R = {depth, plane, score, nghbr};
  memset(depth, 0, sizeof(float) * (size_t)W * H);
  memset(plane, 0, sizeof(float) * 3 * (size_t)W * H);
  memset(score, 0, sizeof(float) * (size_t)W * H);
  memset(nghbr, 0, sizeof(int32_t) * (size_t)W * H);
  const int hpz = V.hpz;
  rng_t rng = {seed};
  for (int i = hpz; i < H - hpz; ++i)
    for (int j = hpz; j < W - hpz; ++j) {
      const float dep = expf(uniform_ab(&rng, (float)log(min_depth), (float)log(max_depth)));
      const float nrm[3] = {uniform_ab(&rng, -1, 1), uniform_ab(&rng, -1, 1), -1};
      float pl[3], s;
      int nb;
      plane_from_depth_normal((float)j, (float)i, V.Kinv[0], dep, nrm, pl);
      if (sample) {
        nb = uniform_int(&rng, n > 1 ? 1 : 0, n > 1 ? n - 1 : 0);
        s = or_plane_image_score_v(&V, i, j, pl, nb);
      } else {
        plane_score(&V, i, j, pl, &s, &nb);
      }
      assign(&R, W, i, j, dep, pl, s, nb);
    }
  const float min_var = min_patch_sd * min_patch_sd;
  for (int i = hpz; i < H - hpz; ++i)
    for (int j = hpz; j < W - hpz; ++j)
      if (masks[(size_t)i * W + j] == 0 || patch_variance(&V, i, j) < min_var) {
        const float z[3] = {0, 0, 0};
        assign(&R, W, i, j, 0.0f, z, 0.0f, 0);
      }
  for (int hp = 0; hp < half_passes; ++hp)
    for (int i = hpz; i < H - hpz; ++i)
      for (int j = hpz + ((i + hp + hpz) & 1); j < W - hpz; j += 2)
        redblack_update(&V, &R, i, j, sample, &rng);
  post_process(&R, W, H);
  views_free(&V);
  return 0;
}

/* ComputePlaneScore for every interior pixel with the given planes. */
int or_score_planes(int n, const double* K, const double* Rm, const double* t,
                    const uint8_t* images, int W, int H, int patch, const float* planes,
                    float* score, int32_t* nghbr) {
  views_t V;
  views_init(&V, n, K, Rm, t, images, NULL, W, H, patch);
  for (int i = 0; i < H; ++i)
    for (int j = 0; j < W; ++j) {
      size_t p = (size_t)i * W + j;
      score[p] = 0.0f;
      nghbr[p] = 0;
      if (i < V.hpz || i >= H - V.hpz || j < V.hpz || j >= W - V.hpz) continue;
      float s;
      int nb;
      plane_score(&V, i, j, planes + 3 * p, &s, &nb);
      score[p] = s;
      nghbr[p] = nb;
    }
  views_free(&V);
  return 0;
}

/* Exact 5x5 median, replicated border (cv::medianBlur, CV_32F, ksize 5). */
static int cmp_float(const void* a, const void* b) {
  float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}
void or_median5(const float* src, float* dst, int W, int H) {
  float win[25];
  for (int i = 0; i < H; ++i)
    for (int j = 0; j < W; ++j) {
      int c = 0;
      for (int di = -2; di <= 2; ++di)
        for (int dj = -2; dj <= 2; ++dj) {
          int ii = i + di < 0 ? 0 : (i + di > H - 1 ? H - 1 : i + di);
          int jj = j + dj < 0 ? 0 : (j + dj > W - 1 ? W - 1 : j + dj);
          win[c++] = src[(size_t)ii * W + jj];
        }
      qsort(win, 25, sizeof(float), cmp_float);
      dst[(size_t)i * W + j] = win[12];
    }
}

/* ------------------------------------------------------------------ cleaner
 * DepthmapCleaner::Clean (depthmap.cc:524-555). */
static void backproject(double x, double y, double depth, const double* K, const double* R,
                        const double* t, double out[3]) {
  double Ki[9], M[9], q[3] = {x, y, 1.0}, p[3], Rt[9];
  or_inv3(K, Ki);
  for (int k = 0; k < 9; ++k) M[k] = Ki[k] * depth;
  m3_vec(M, q, p);
  for (int k = 0; k < 3; ++k) p[k] = p[k] - t[k];
  m3_t(R, Rt);
  m3_vec(Rt, p, out);
}
static void project(const double X[3], const double* K, const double* R, const double* t,
                    double out[3]) {
  double p[3];
  m3_vec(R, X, p);
  for (int k = 0; k < 3; ++k) p[k] = p[k] + t[k];
  m3_vec(K, p, out);
}

int or_clean(int n, const double* K, const double* R, const double* t, const float* depths,
             int W, int H, float thr, int min_views, float* out) {
  for (int i = 0; i < H; ++i)
    for (int j = 0; j < W; ++j) {
      size_t p = (size_t)i * W + j;
      float depth = depths[p];
      double Xd[3];
      backproject(j, i, depth, K, R, t, Xd);
      double X[3] = {(float)Xd[0], (float)Xd[1], (float)Xd[2]};
      int consistent = 1;
      for (int o = 1; o < n; ++o) {
        double rd[3];
        project(X, K + 9 * o, R + 9 * o, t + 3 * o, rd);
        float r0 = (float)rd[0], r1 = (float)rd[1], r2 = (float)rd[2];
        if (r2 < 1e-8 || isnan(r2)) continue;
        float u = r0 / r2, v = r1 / r2;
        float dr = bilinear_f32(depths + (size_t)o * W * H, W, H, v, u);
        if (fabsf(dr - r2) < r2 * thr) consistent++;
      }
      out[p] = (consistent >= min_views) ? depths[p] : 0;
    }
  return 0;
}

/* ------------------------------------------------------------------- pruner
 * DepthmapPruner::Prune (depthmap.cc:577-637).  Writes at most `capacity`
 * points; returns the number of kept points. */
static void normalize3f(const float* v, float out[3]) {
  double s = 0;
  for (int k = 0; k < 3; ++k) {
    double x = v[k];
    s += x * x;
  }
  double nv = sqrt(s);
  double a = nv ? 1. / nv : 0.;
  for (int k = 0; k < 3; ++k) out[k] = (float)(v[k] * a);
}

long or_prune(int n, const double* K, const double* R, const double* t, const float* depths,
              const float* planes, const uint8_t* colors, const uint8_t* labels, int W, int H,
              float thr, float* points, float* normals, uint8_t* colors_out,
              uint8_t* labels_out, long capacity) {
  float Rinv[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Rinv[3 * i + j] = (float)R[3 * j + i];
  long count = 0;
  const size_t N = (size_t)W * H;
  for (int i = 0; i < H; ++i)
    for (int j = 0; j < W; ++j) {
      size_t p = (size_t)i * W + j;
      float depth = depths[p];
      if (depth <= 0) continue;
      float nrm[3];
      normalize3f(planes + 3 * p, nrm);
      float area = (float)(-nrm[2] / depth * K[0]);
      double Xd[3];
      backproject(j, i, depth, K, R, t, Xd);
      float Xf[3] = {(float)Xd[0], (float)Xd[1], (float)Xd[2]};
      double X[3] = {Xf[0], Xf[1], Xf[2]};
      int keep = 1;
      for (int o = 1; o < n && keep; ++o) {
        double rp[3];
        project(X, K + 9 * o, R + 9 * o, t + 3 * o, rp);
        if (rp[2] < 1e-8 || isnan(rp[2])) continue;
        int64_t iu = (int64_t)(rp[0] / rp[2] + 0.5);
        int64_t iv = (int64_t)(rp[1] / rp[2] + 0.5);
        double dop = rp[2];
        int ii = (int)iv, jj = (int)iu;
        if (!(ii >= 0 && ii < H && jj >= 0 && jj < W)) continue;
        size_t q = (size_t)ii * W + jj;
        float dr = depths[o * N + q];
        if (dr > (1 - thr) * dop) {
          float no[3];
          normalize3f(planes + 3 * (o * N + q), no);
          if ((dr == 0.0) || ((-no[2] / dr) * K[9 * o] > area)) keep = 0;
        }
      }
      if (!keep) continue;
      if (count < capacity) {
        float rn[3];
        for (int a = 0; a < 3; ++a) {
          float s = 0.0f;
          for (int b = 0; b < 3; ++b) s += Rinv[3 * a + b] * nrm[b];
          rn[a] = s;
        }
        for (int a = 0; a < 3; ++a) {
          points[3 * count + a] = Xf[a];
          normals[3 * count + a] = rn[a];
          colors_out[3 * count + a] = colors[3 * p + a];
        }
        labels_out[count] = labels[p];
      }
      count++;
    }
  return count;
}
