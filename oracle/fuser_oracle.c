/* DepthmapFuser::Fuse restated in C.  TEST INFRASTRUCTURE ONLY.
 *
 * Follows opensfm/src/lib/dense/src/fuser.cc:115-372 (per-pixel fusion;
 * or_sor below restates the statistical outlier removal of 374-482) with the reference's
 * single-thread order: primary views in index order, pixels in raster
 * order, each fused pixel marking itself and the source pixels it used.
 * Arithmetic is FP32 with every operation rounded by itself, in the order
 * the reference's expressions are written (the reference's own build may
 * contract products into FMAs; this file fixes the order without
 * contraction, and the 3x3 inverse in Eigen's cofactor order).  Parity is
 * unpinned by the reference's outputs: it needs Eigen and vlfeat, which are
 * absent here.  The library's fuser must match this file bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct {
  const double* K;      /* 3x3 row-major */
  const double* R;      /* 3x3 row-major */
  const double* t;      /* 3 */
  int W, H;
  const float* depth;   /* [H][W] */
  const float* normal;  /* [H][W][3] */
  const uint8_t* color; /* [H][W][3] */
  const uint8_t* mask;  /* [H][W] or NULL */
  const int* nbrs;
  int n_nbrs;
  int primary;
} or_fuse_view;

typedef struct {
  float K[9], Kinv[9], R[9], t[3];
} fcam;

/* Eigen's 3x3 inverse: cofactors cof(i,j) = m(i1,j1) m(i2,j2) - m(i1,j2)
 * m(i2,j1) with i1 = i+1, i2 = i+2, j1 = j+1, j2 = j+2 (mod 3), det from the
 * first column, inverse(j,i) = cof(i,j) * (1 / det). */
static void inv3f(const float* m, float* o) {
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

static void make_cam(const or_fuse_view* v, fcam* c) {
  for (int i = 0; i < 9; ++i) {
    c->K[i] = (float)v->K[i];
    c->R[i] = (float)v->R[i];
  }
  for (int i = 0; i < 3; ++i) c->t[i] = (float)v->t[i];
  inv3f(c->K, c->Kinv);
}

/* M x */
static void mv(const float* m, float x, float y, float z, float* o) {
  o[0] = (m[0] * x + m[1] * y) + m[2] * z;
  o[1] = (m[3] * x + m[4] * y) + m[5] * z;
  o[2] = (m[6] * x + m[7] * y) + m[8] * z;
}
/* M^T x */
static void mtv(const float* m, float x, float y, float z, float* o) {
  o[0] = (m[0] * x + m[3] * y) + m[6] * z;
  o[1] = (m[1] * x + m[4] * y) + m[7] * z;
  o[2] = (m[2] * x + m[5] * y) + m[8] * z;
}
/* R^T (d K^-1 (u, v, 1) - t) */
static void backproject(const fcam* c, float d, float u, float v, float* o) {
  float m[9], q[3];
  for (int i = 0; i < 9; ++i) m[i] = d * c->Kinv[i];
  mv(m, u, v, 1.0f, q);
  mtv(c->R, q[0] - c->t[0], q[1] - c->t[1], q[2] - c->t[2], o);
}
/* K (R X + t) */
static void project(const fcam* c, const float* X, float* o) {
  float p[3];
  mv(c->R, X[0], X[1], X[2], p);
  mv(c->K, p[0] + c->t[0], p[1] + c->t[1], p[2] + c->t[2], o);
}

/* BilinearDepth (fuser.cc:95-113) over foundation::BilinearInterpolation. */
static float bilinear_depth(const float* d, int W, int H, float u, float v) {
  const int x0 = (int)floorf(u), y0 = (int)floorf(v), x1 = x0 + 1, y1 = y0 + 1;
  if (x0 < 0 || y0 < 0 || x1 >= W || y1 >= H) return -1.0f;
  if (d[y0 * W + x0] <= 0.0f || d[y0 * W + x1] <= 0.0f || d[y1 * W + x0] <= 0.0f ||
      d[y1 * W + x1] <= 0.0f)
    return -1.0f;
  if (u < 0.0f || u >= W - 1 || v < 0.0f || v >= H - 1) return -1.0f;
  const int ix = (int)u, iy = (int)v;
  const float dx = u - ix, dy = v - iy;
  const float v0 = (1 - dx) * d[iy * W + ix] + dx * d[iy * W + ix + 1];
  const float v1 = (1 - dx) * d[(iy + 1) * W + ix] + dx * d[(iy + 1) * W + ix + 1];
  return (1 - dy) * v0 + dy * v1;
}

static int cmp_f(const void* a, const void* b) {
  const float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}
static int cmp_u8(const void* a, const void* b) {
  return (int)*(const uint8_t*)a - (int)*(const uint8_t*)b;
}
/* VectorMedian (fuser.cc:23-31): the element nth_element puts at n / 2. */
static float median_f(float* v, int n) {
  qsort(v, (size_t)n, sizeof(float), cmp_f);
  return v[n / 2];
}
static uint8_t median_u8(uint8_t* v, int n) {
  qsort(v, (size_t)n, 1, cmp_u8);
  return v[n / 2];
}

long or_fuse(const or_fuse_view* views, int n_views, int min_num_consistent,
             float max_reproj_error_px, float max_depth_error, float max_normal_error_deg,
             int border_margin, float behind_depth_factor, float* out_pts, float* out_nrm,
             uint8_t* out_clr, long capacity) {
  const float max_reproj_sq = max_reproj_error_px * max_reproj_error_px;
  const float min_cos = cosf(max_normal_error_deg * (float)M_PI / 180.0f);
  const int bm = border_margin < 0 ? 0 : border_margin;
  float behind = behind_depth_factor;
  if (behind < 0.0f) behind = 0.0f;
  if (behind > 1.0f) behind = 1.0f;
  fcam* cams = (fcam*)malloc(sizeof(fcam) * (size_t)n_views);
  uint8_t** fused = (uint8_t**)malloc(sizeof(uint8_t*) * (size_t)n_views);
  for (int v = 0; v < n_views; ++v) {
    make_cam(&views[v], &cams[v]);
    fused[v] = (uint8_t*)calloc((size_t)views[v].W * views[v].H, 1);
  }
  int max_obs = 1;
  for (int v = 0; v < n_views; ++v)
    if (1 + views[v].n_nbrs > max_obs) max_obs = 1 + views[v].n_nbrs;
  float* pts = (float*)malloc(sizeof(float) * 3 * (size_t)max_obs);
  float* nrm = (float*)malloc(sizeof(float) * 3 * (size_t)max_obs);
  uint8_t* clr = (uint8_t*)malloc(3 * (size_t)max_obs);
  int* used_v = (int*)malloc(sizeof(int) * (size_t)max_obs);
  int* used_p = (int*)malloc(sizeof(int) * (size_t)max_obs);
  float* comp = (float*)malloc(sizeof(float) * (size_t)max_obs);
  uint8_t* comp8 = (uint8_t*)malloc((size_t)max_obs);
  long count = 0;
  for (int ri = 0; ri < n_views; ++ri) {
    const or_fuse_view* ref = &views[ri];
    if (!ref->primary) continue;
    const fcam* rc = &cams[ri];
    const int rows = ref->H, cols = ref->W;
    for (int r = bm; r < rows - bm; ++r) {
      for (int c = bm; c < cols - bm; ++c) {
        const int rp = r * cols + c;
        if (fused[ri][rp]) continue;
        if (ref->mask && ref->mask[rp] == 0) continue;
        const float rd = ref->depth[rp];
        if (rd <= 0.0f) continue;
        float ref_point[3];
        backproject(rc, rd, (float)c, (float)r, ref_point);
        const float* rn = ref->normal + 3 * (size_t)rp;
        const float nlen = sqrtf((rn[0] * rn[0] + rn[1] * rn[1]) + rn[2] * rn[2]);
        if (nlen < 1e-6f) continue;
        float rnw[3];
        mtv(rc->R, rn[0] / nlen, rn[1] / nlen, rn[2] / nlen, rnw);
        int n_obs = 1, n_used = 0;
        memcpy(pts, ref_point, sizeof(ref_point));
        memcpy(nrm, rnw, sizeof(rnw));
        memcpy(clr, ref->color + 3 * (size_t)rp, 3);
        for (int k = 0; k < ref->n_nbrs; ++k) {
          const int si = ref->nbrs[k];
          if (si < 0 || si >= n_views) continue;
          const or_fuse_view* src = &views[si];
          const fcam* sc = &cams[si];
          float proj[3];
          project(sc, ref_point, proj);
          if (proj[2] < 1e-6f) continue;
          const float su = proj[0] / proj[2], sv = proj[1] / proj[2];
          /* Far outside the image (or NaN): out of bounds, as the reference's
           * int conversion of such values is on x86. */
          if (!(fabsf(su) < 1e9f && fabsf(sv) < 1e9f)) continue;
          const int scol = (int)roundf(su), srow = (int)roundf(sv);
          if (scol < bm || scol >= src->W - bm || srow < bm || srow >= src->H - bm) continue;
          const int sp = srow * src->W + scol;
          if (src->mask && src->mask[sp] == 0) continue;
          if (fused[si][sp]) continue;
          float sd = bilinear_depth(src->depth, src->W, src->H, su, sv);
          if (sd <= 0.0f) {
            sd = src->depth[sp];
            if (sd <= 0.0f) continue;
          }
          const float front = max_depth_error * proj[2];
          const float back = front * behind;
          const float diff = sd - proj[2];
          if (diff > front || diff < -back) continue;
          float spt[3], rep[3];
          backproject(sc, sd, (float)scol, (float)srow, spt);
          project(rc, spt, rep);
          if (rep[2] < 1e-6f) continue;
          const float ex = rep[0] / rep[2] - (float)c, ey = rep[1] / rep[2] - (float)r;
          if (ex * ex + ey * ey > max_reproj_sq) continue;
          const float* sn = src->normal + 3 * (size_t)sp;
          const float slen = sqrtf((sn[0] * sn[0] + sn[1] * sn[1]) + sn[2] * sn[2]);
          if (slen < 1e-6f) continue;
          float snw[3];
          mtv(sc->R, sn[0] / slen, sn[1] / slen, sn[2] / slen, snw);
          const float cosang = (rnw[0] * snw[0] + rnw[1] * snw[1]) + rnw[2] * snw[2];
          if (cosang < min_cos) continue;
          memcpy(pts + 3 * n_obs, spt, sizeof(spt));
          memcpy(nrm + 3 * n_obs, snw, sizeof(snw));
          memcpy(clr + 3 * n_obs, src->color + 3 * (size_t)sp, 3);
          ++n_obs;
          used_v[n_used] = si;
          used_p[n_used] = sp;
          ++n_used;
        }
        if (n_obs < min_num_consistent) continue;
        if (count >= capacity) goto done;
        for (int d = 0; d < 3; ++d) {
          for (int k = 0; k < n_obs; ++k) comp[k] = pts[3 * k + d];
          out_pts[3 * count + d] = median_f(comp, n_obs);
        }
        float mn[3];
        for (int d = 0; d < 3; ++d) {
          for (int k = 0; k < n_obs; ++k) comp[k] = nrm[3 * k + d];
          mn[d] = median_f(comp, n_obs);
        }
        const float ml = sqrtf((mn[0] * mn[0] + mn[1] * mn[1]) + mn[2] * mn[2]);
        if (ml > 1e-6f)
          for (int d = 0; d < 3; ++d) mn[d] = mn[d] / ml;
        memcpy(out_nrm + 3 * count, mn, sizeof(mn));
        for (int d = 0; d < 3; ++d) {
          for (int k = 0; k < n_obs; ++k) comp8[k] = clr[3 * k + d];
          out_clr[3 * count + d] = median_u8(comp8, n_obs);
        }
        ++count;
        fused[ri][rp] = 1;
        for (int k = 0; k < n_used; ++k) fused[used_v[k]][used_p[k]] = 1;
      }
    }
  }
done:
  for (int v = 0; v < n_views; ++v) free(fused[v]);
  free(fused);
  free(cams);
  free(pts);
  free(nrm);
  free(clr);
  free(used_v);
  free(used_p);
  free(comp);
  free(comp8);
  return count;
}

/* Statistical outlier removal (fuser.cc:374-482).  The reference finds the
 * K + 1 nearest neighbours of every point with a vlfeat kd-forest of one
 * tree and vlfeat's default comparison limit 0, which vlfeat defines as an
 * exact search; the distances are vlfeat's float L2, the squared distance
 * summed over x, y, z in that order.  Skipping the point itself leaves the
 * K smallest distances to other points, so that set is found here by brute
 * force (O(N^2): small inputs only), summed as float square roots in
 * ascending order and divided by K.  Mean and variance of those means are
 * accumulated in double in point order; points with a mean at or below
 * mean + factor * std (rounded to float) are kept.  keep[i] is set to 0/1;
 * mean_knn (optional) receives the per-point means.  Returns the kept count,
 * or n (all kept) when k <= 0 or n <= k + 1, as the reference skips the step. */
long or_sor(const float* pts, long n, int k, float factor, uint8_t* keep, float* mean_knn) {
  if (k <= 0 || n <= (long)k + 1) {
    for (long i = 0; i < n; ++i) keep[i] = 1;
    return n;
  }
  float* best = (float*)malloc(sizeof(float) * (size_t)k);
  float* mk = (float*)malloc(sizeof(float) * (size_t)n);
  for (long i = 0; i < n; ++i) {
    const float* q = pts + 3 * i;
    int cnt = 0;
    for (long j = 0; j < n; ++j) {
      if (j == i) continue;
      const float* p = pts + 3 * j;
      const float dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
      float d2 = dx * dx;
      d2 = d2 + dy * dy;
      d2 = d2 + dz * dz;
      if (cnt == k && !(d2 < best[k - 1])) continue;
      int m = cnt < k ? cnt++ : k - 1;
      while (m > 0 && best[m - 1] > d2) {
        best[m] = best[m - 1];
        --m;
      }
      best[m] = d2;
    }
    float sum = 0.0f;
    for (int m = 0; m < k; ++m) sum += sqrtf(best[m]);
    mk[i] = sum / (float)k;
  }
  double sum_d = 0.0, sum_d2 = 0.0;
  for (long i = 0; i < n; ++i) {
    const double d = mk[i];
    if (d < 1e20f) {
      sum_d += d;
      sum_d2 += d * d;
    }
  }
  const double mean_d = sum_d / (double)n;
  const double var_d = sum_d2 / (double)n - mean_d * mean_d;
  const double std_d = sqrt(var_d > 0.0 ? var_d : 0.0);
  const float threshold = (float)(mean_d + factor * std_d);
  long kept = 0;
  for (long i = 0; i < n; ++i) {
    keep[i] = mk[i] <= threshold;
    kept += keep[i];
    if (mean_knn) mean_knn[i] = mk[i];
  }
  free(best);
  free(mk);
  return kept;
}
