/* SVOFuser (TSDF fusion into a sparse voxel hash) restated in C.
 * TEST INFRASTRUCTURE ONLY.
 *
 * Follows opensfm/src/lib/dense/src/svo_fuser.cc:52-183 (CountVoxels, Fuse),
 * src/svo_opencl.cc:169-277 and 527-630 (camera set-up, integration and
 * extraction launches) and the kernels of svo_opencl_kernels.h:187-651
 * (svo_integrate, svo_count, svo_extract_points).  The reference runs them
 * as OpenCL kernels, unavailable here; parity is unpinned by the reference's
 * outputs and this file fixes the arithmetic instead: FP32, every operation
 * rounded by itself in the order the kernel source writes it (no
 * contraction), length() as sqrtf((x*x + y*y) + z*z), correctly rounded
 * division and square root.  The library's SVO fuser must match this file
 * bit for bit.
 *
 * The reference accumulates fixed-point integers with atomic adds, so a
 * voxel's sums do not depend on the order of the contributions; here they
 * are collected, sorted by voxel and summed with 32-bit wrap-around.  Its
 * points leave in the order of an atomic counter over hash slots, which is
 * not reproducible; this file and the library emit them in ascending voxel
 * order (x, then y, then z, all signed) and, per voxel, +X, +Y, +Z.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SVO_FP_SCALE 32768
#define SVO_WEIGHT_SCALE 128
#define SVO_COS_THETA_MIN 0.15f

typedef struct {
  const double* K; /* 3x3 row-major */
  const double* R; /* 3x3 row-major */
  const double* t; /* 3 */
  int W, H;
  const float* depth;   /* [H][W] */
  const float* normal;  /* [H][W][3] or NULL */
  const uint8_t* color; /* [H][W][3] or NULL */
  const uint8_t* mask;  /* [H][W] or NULL */
  const float* weight;  /* [H][W] or NULL */
} or_svo_view;

typedef struct {
  float Kinv[9], Rinv[9], R[9], t[3], cp[3];
} svo_cam;

/* Eigen's 3x3 inverse (cofactors, determinant from the first column). */
static void svo_inv3(const float* m, float* o) {
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

/* svo_opencl.cc:213-226: Kinv = K^-1, Rinv = R^T, cam_pos = -Rinv t, from
 * the float casts of K, R, t. */
static void svo_make_cam(const or_svo_view* v, svo_cam* c) {
  float K[9];
  for (int i = 0; i < 9; ++i) {
    K[i] = (float)v->K[i];
    c->R[i] = (float)v->R[i];
  }
  for (int i = 0; i < 3; ++i) c->t[i] = (float)v->t[i];
  svo_inv3(K, c->Kinv);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) c->Rinv[3 * i + j] = c->R[3 * j + i];
  for (int i = 0; i < 3; ++i)
    c->cp[i] = ((-c->Rinv[3 * i] * c->t[0]) + (-c->Rinv[3 * i + 1] * c->t[1])) +
               (-c->Rinv[3 * i + 2] * c->t[2]);
}

/* A voxel coordinate as a 64-bit key that sorts as (x, y, z) signed. */
static uint64_t svo_key(int kx, int ky, int kz) {
  return ((uint64_t)(uint32_t)(kx + 32768) << 48) | ((uint64_t)(uint32_t)(ky + 32768) << 32) |
         (uint64_t)((uint32_t)kz ^ 0x80000000u);
}

typedef struct {
  uint64_t key;
  int32_t v[9]; /* count, weight, tsdf, nx, ny, nz, r, g, b (weighted) */
} svo_contrib;

typedef struct {
  svo_contrib* a;
  size_t n, cap;
} svo_list;

static int svo_push(svo_list* l, const svo_contrib* c) {
  if (l->n == l->cap) {
    const size_t nc = l->cap ? 2 * l->cap : 4096;
    svo_contrib* na = (svo_contrib*)realloc(l->a, nc * sizeof(svo_contrib));
    if (!na) return -1;
    l->a = na;
    l->cap = nc;
  }
  l->a[l->n++] = *c;
  return 0;
}

typedef struct {
  float voxel_size, trunc, inv_vs;
  int has_bbox;
  int bmin[3], bmax[3];
} svo_params;

/* The per-pixel march of svo_integrate (counting = 0) or svo_count
 * (counting = 1): every voxel sample of the truncation band is appended. */
static int svo_march(const or_svo_view* v, const svo_cam* cam, const svo_params* p, int counting,
                     svo_list* out) {
  for (int r = 0; r < v->H; ++r)
    for (int c = 0; c < v->W; ++c) {
      const size_t idx = (size_t)r * v->W + c;
      if (v->mask && v->mask[idx] == 0) continue;
      const float d = v->depth[idx];
      if (!(d > 0.0f)) continue;
      const float uc = (float)c, vr = (float)r;
      const float pc[3] = {d * ((cam->Kinv[0] * uc + cam->Kinv[1] * vr) + cam->Kinv[2]),
                           d * ((cam->Kinv[3] * uc + cam->Kinv[4] * vr) + cam->Kinv[5]),
                           d * ((cam->Kinv[6] * uc + cam->Kinv[7] * vr) + cam->Kinv[8])};
      const float df[3] = {pc[0] - cam->t[0], pc[1] - cam->t[1], pc[2] - cam->t[2]};
      float pw[3], ray[3];
      for (int i = 0; i < 3; ++i)
        pw[i] = (cam->Rinv[3 * i] * df[0] + cam->Rinv[3 * i + 1] * df[1]) +
                cam->Rinv[3 * i + 2] * df[2];
      for (int i = 0; i < 3; ++i) ray[i] = pw[i] - cam->cp[i];
      const float ray_len = sqrtf((ray[0] * ray[0] + ray[1] * ray[1]) + ray[2] * ray[2]);
      if (ray_len < 1e-8f) continue;
      if (ray_len * 1.2e-7f >= p->voxel_size) continue;
      for (int i = 0; i < 3; ++i) ray[i] = ray[i] / ray_len;
      const float ts = ray_len - p->trunc;
      const float t_start = ts > 0.0f ? ts : 0.0f;
      const float t_end = ray_len + p->trunc;
      int nfp[3] = {0, 0, 0}, rgb[3] = {0, 0, 0}, w_int = 1;
      if (!counting) {
        if (v->normal) {
          const float* nc = v->normal + 3 * idx;
          const float nlen = sqrtf((nc[0] * nc[0] + nc[1] * nc[1]) + nc[2] * nc[2]);
          if (nlen > 1e-6f) {
            const float n[3] = {nc[0] / nlen, nc[1] / nlen, nc[2] / nlen};
            float nw[3];
            for (int i = 0; i < 3; ++i)
              nw[i] = (cam->Rinv[3 * i] * n[0] + cam->Rinv[3 * i + 1] * n[1]) +
                      cam->Rinv[3 * i + 2] * n[2];
            for (int i = 0; i < 3; ++i) nfp[i] = (int)(nw[i] * (float)SVO_FP_SCALE);
            const float cs = fabsf((ray[0] * nw[0] + ray[1] * nw[1]) + ray[2] * nw[2]);
            if (cs < SVO_COS_THETA_MIN) continue; /* grazing */
          }
        }
        if (v->color)
          for (int i = 0; i < 3; ++i) rgb[i] = (int)v->color[3 * idx + i];
        float wf = 1.0f;
        if (v->weight) wf = wf * v->weight[idx];
        const float ws = wf * (float)SVO_WEIGHT_SCALE;
        /* (int) of the scaled weight, saturating (NaN counts as 0), then
         * clamped to [1, 4 * WEIGHT_SCALE]. */
        int wi = ws != ws ? 0 : (ws >= 2147483520.0f ? 2147483647 : (ws <= -2147483648.0f ? (-2147483647 - 1) : (int)ws));
        w_int = wi < 1 ? 1 : (wi > 4 * SVO_WEIGHT_SCALE ? 4 * SVO_WEIGHT_SCALE : wi);
      }
      for (float tt = t_start; tt <= t_end; tt += p->voxel_size) {
        float s[3];
        int k[3], skip = 0;
        for (int i = 0; i < 3; ++i) {
          s[i] = cam->cp[i] + tt * ray[i];
          const float f = floorf(s[i] * p->inv_vs);
          if (!(f >= -2147483648.0f && f < 2147483648.0f)) skip = 1;
          k[i] = skip ? 0 : (int)f;
        }
        if (skip) continue;
        if (k[0] < -32768 || k[0] > 32766 || k[1] < -32768 || k[1] > 32766) continue;
        if (p->has_bbox && (k[0] < p->bmin[0] || k[0] > p->bmax[0] || k[1] < p->bmin[1] ||
                            k[1] > p->bmax[1] || k[2] < p->bmin[2] || k[2] > p->bmax[2]))
          continue;
        const float ctr[3] = {((float)k[0] + 0.5f) * p->voxel_size,
                              ((float)k[1] + 0.5f) * p->voxel_size,
                              ((float)k[2] + 0.5f) * p->voxel_size};
        const float zc =
            ((cam->R[6] * ctr[0] + cam->R[7] * ctr[1]) + cam->R[8] * ctr[2]) + cam->t[2];
        if (zc <= 0.0f) continue;
        const float sdf = d - zc;
        if (sdf < -p->trunc) continue;
        svo_contrib e;
        e.key = svo_key(k[0], k[1], k[2]);
        memset(e.v, 0, sizeof(e.v));
        if (!counting) {
          const float q = sdf / p->trunc;
          const float tsdf = q < 1.0f ? q : 1.0f;
          const int tfp = (int)(tsdf * (float)SVO_FP_SCALE);
          e.v[0] = 1;
          e.v[1] = w_int;
          e.v[2] = (int32_t)((uint32_t)tfp * (uint32_t)w_int);
          for (int i = 0; i < 3; ++i) e.v[3 + i] = (int32_t)((uint32_t)nfp[i] * (uint32_t)w_int);
          for (int i = 0; i < 3; ++i) e.v[6 + i] = rgb[i] * w_int;
        }
        if (svo_push(out, &e)) return -1;
      }
    }
  return 0;
}

static int svo_cmp(const void* a, const void* b) {
  const uint64_t x = ((const svo_contrib*)a)->key, y = ((const svo_contrib*)b)->key;
  return x < y ? -1 : (x > y ? 1 : 0);
}

static void svo_bbox(const svo_params* p, const float* bmin, const float* bmax, svo_params* o) {
  *o = *p;
  o->has_bbox = bmin && bmax;
  if (o->has_bbox)
    for (int i = 0; i < 3; ++i) {
      o->bmin[i] = (int)floorf(bmin[i] * p->inv_vs);
      o->bmax[i] = (int)ceilf(bmax[i] * p->inv_vs);
    }
}

/* CountVoxels (svo_fuser.cc:52-106): the number of distinct voxels the
 * counting march touches (no grazing test, no values). */
long or_svo_count(const or_svo_view* views, int n_views, float voxel_size, float trunc_factor,
                  const float* bbox_min, const float* bbox_max) {
  svo_params p0 = {voxel_size, trunc_factor * voxel_size, 1.0f / voxel_size, 0, {0}, {0}}, p;
  svo_bbox(&p0, bbox_min, bbox_max, &p);
  svo_list l = {0};
  for (int v = 0; v < n_views; ++v) {
    svo_cam cam;
    svo_make_cam(&views[v], &cam);
    if (svo_march(&views[v], &cam, &p, 1, &l)) {
      free(l.a);
      return -1;
    }
  }
  qsort(l.a, l.n, sizeof(svo_contrib), svo_cmp);
  long u = 0;
  for (size_t i = 0; i < l.n; ++i)
    if (i == 0 || l.a[i].key != l.a[i - 1].key) ++u;
  free(l.a);
  return u;
}

static float svo_clampf(float x, float lo, float hi) {
  const float m = x > lo ? x : lo;
  return m < hi ? m : hi;
}

/* Fuse (svo_fuser.cc:108-183) after CountVoxels returned `count`: the
 * integration, then svo_extract_points over the voxels in ascending order.
 * Writes at most `capacity` points; returns how many the reference would
 * emit (at most its max_output = table capacity / 4), or -1 on allocation
 * failure. */
long or_svo_fuse(const or_svo_view* views, int n_views, float voxel_size, float trunc_factor,
                 float min_weight, const float* bbox_min, const float* bbox_max, long count,
                 float* out_pts, float* out_nrm, uint8_t* out_clr, long capacity) {
  svo_params p0 = {voxel_size, trunc_factor * voxel_size, 1.0f / voxel_size, 0, {0}, {0}}, p;
  svo_bbox(&p0, bbox_min, bbox_max, &p);
  svo_list l = {0};
  for (int v = 0; v < n_views; ++v) {
    svo_cam cam;
    svo_make_cam(&views[v], &cam);
    if (svo_march(&views[v], &cam, &p, 0, &l)) {
      free(l.a);
      return -1;
    }
  }
  qsort(l.a, l.n, sizeof(svo_contrib), svo_cmp);
  /* Reduce to one entry per voxel, sums with 32-bit wrap-around. */
  size_t nu = 0;
  for (size_t i = 0; i < l.n; ++i) {
    if (nu > 0 && l.a[nu - 1].key == l.a[i].key) {
      for (int f = 0; f < 9; ++f)
        l.a[nu - 1].v[f] = (int32_t)((uint32_t)l.a[nu - 1].v[f] + (uint32_t)l.a[i].v[f]);
    } else {
      l.a[nu++] = l.a[i];
    }
  }
  /* The reference's table holds max(2 count, 2^20) slots rounded up to a
   * power of two and emits at most a quarter of that. */
  uint64_t want = (uint64_t)count * 2;
  if (want < (1u << 20)) want = 1u << 20;
  uint64_t cap = 1;
  while (cap < want) cap <<= 1;
  const long max_output = (long)(cap / 4);
  const float mws = min_weight * (float)SVO_WEIGHT_SCALE;
  long n = 0;
  for (size_t i = 0; i < nu && n < max_output; ++i) {
    const svo_contrib* a = &l.a[i];
    if (a->v[0] == 0) continue;
    const float sw_a = (float)a->v[1];
    if (sw_a < mws) continue;
    const int kx = (int)((a->key >> 48) & 0xFFFF) - 32768;
    const int ky = (int)((a->key >> 32) & 0xFFFF) - 32768;
    const int kz = (int)((uint32_t)a->key ^ 0x80000000u);
    const float inv_sw_a = 1.0f / sw_a;
    const float inv_fp_sw_a = inv_sw_a / (float)SVO_FP_SCALE;
    const float tsdf_a = (float)a->v[2] * inv_fp_sw_a;
    const float na[3] = {(float)a->v[3] * inv_fp_sw_a, (float)a->v[4] * inv_fp_sw_a,
                         (float)a->v[5] * inv_fp_sw_a};
    const float ca[3] = {(float)a->v[6] * inv_sw_a, (float)a->v[7] * inv_sw_a,
                         (float)a->v[8] * inv_sw_a};
    for (int d = 0; d < 3 && n < max_output; ++d) {
      const int nx = kx + (d == 0), ny = ky + (d == 1), nz = kz + (d == 2);
      if (nx > 32766 || ny > 32766) continue; /* not storable: never found */
      const uint64_t kb = svo_key(nx, ny, nz);
      size_t lo = 0, hi = nu;
      while (lo < hi) {
        const size_t mid = (lo + hi) / 2;
        if (l.a[mid].key < kb)
          lo = mid + 1;
        else
          hi = mid;
      }
      if (lo >= nu || l.a[lo].key != kb) continue;
      const svo_contrib* b = &l.a[lo];
      const float sw_b = (float)b->v[1];
      if (sw_b < mws) continue;
      const float inv_sw_b = 1.0f / sw_b;
      const float inv_fp_sw_b = inv_sw_b / (float)SVO_FP_SCALE;
      const float tsdf_b = (float)b->v[2] * inv_fp_sw_b;
      if ((tsdf_a > 0.0f) == (tsdf_b > 0.0f)) continue;
      if (tsdf_a == 0.0f || tsdf_b == 0.0f) continue;
      const float t = svo_clampf(tsdf_a / (tsdf_a - tsdf_b), 0.0f, 1.0f);
      const int ka[3] = {kx, ky, kz}, kbv[3] = {nx, ny, nz};
      float pt[3], nn[3];
      for (int i = 0; i < 3; ++i) {
        const float pa = ((float)ka[i] + 0.5f) * voxel_size;
        const float pb = ((float)kbv[i] + 0.5f) * voxel_size;
        pt[i] = pa + t * (pb - pa);
      }
      const float nb[3] = {(float)b->v[3] * inv_fp_sw_b, (float)b->v[4] * inv_fp_sw_b,
                           (float)b->v[5] * inv_fp_sw_b};
      for (int i = 0; i < 3; ++i) nn[i] = na[i] + t * (nb[i] - na[i]);
      const float nlen = sqrtf((nn[0] * nn[0] + nn[1] * nn[1]) + nn[2] * nn[2]);
      if (nlen > 1e-6f)
        for (int i = 0; i < 3; ++i) nn[i] = nn[i] / nlen;
      const float cb[3] = {(float)b->v[6] * inv_sw_b, (float)b->v[7] * inv_sw_b,
                           (float)b->v[8] * inv_sw_b};
      if (n < capacity) {
        for (int i = 0; i < 3; ++i) {
          out_pts[3 * n + i] = pt[i];
          out_nrm[3 * n + i] = nn[i];
          out_clr[3 * n + i] = (uint8_t)svo_clampf(ca[i] + t * (cb[i] - ca[i]), 0.0f, 255.0f);
        }
      }
      ++n;
    }
  }
  free(l.a);
  return n;
}
