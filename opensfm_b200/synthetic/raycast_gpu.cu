// GPU version of raycast.c (same scene model, same hash / noise / shading),
// used to render the many seeded scenes the learned initialisation trains
// on.  One thread per pixel; geometry in double precision as on the CPU.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace {

struct Scene {
  const double* boxes;
  int n_boxes;
  int ground;
  double ground_half;
  int terrain;
  double terrain_amp, terrain_scale;
  uint32_t terrain_seed;
  int terrain_octaves;
  uint32_t tex_seed;
  double tex_freq;
  int tex_octaves;
  double contrast;
  double sky;
};

__device__ uint32_t hash3(int32_t x, int32_t y, int32_t z, uint32_t seed) {
  uint32_t h = seed ^ 0x9E3779B9u;
  h ^= (uint32_t)x * 0x85EBCA6Bu;
  h = (h << 13) | (h >> 19);
  h ^= (uint32_t)y * 0xC2B2AE35u;
  h = (h << 17) | (h >> 15);
  h ^= (uint32_t)z * 0x27D4EB2Fu;
  h ^= h >> 16;
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h;
}
__device__ double fade(double t) { return t * t * t * (t * (t * 6.0 - 15.0) + 10.0); }
__device__ double lerp(double a, double b, double t) { return a + (b - a) * t; }

__device__ double value_noise3(double x, double y, double z, uint32_t seed) {
  double fx = floor(x), fy = floor(y), fz = floor(z);
  int32_t ix = (int32_t)fx, iy = (int32_t)fy, iz = (int32_t)fz;
  double tx = fade(x - fx), ty = fade(y - fy), tz = fade(z - fz);
  double c[8];
  for (int k = 0; k < 8; ++k)
    c[k] = (hash3(ix + (k & 1), iy + ((k >> 1) & 1), iz + (k >> 2), seed) >> 8) *
           (1.0 / 16777216.0);
  double x00 = lerp(c[0], c[1], tx), x10 = lerp(c[2], c[3], tx);
  double x01 = lerp(c[4], c[5], tx), x11 = lerp(c[6], c[7], tx);
  return lerp(lerp(x00, x10, ty), lerp(x01, x11, ty), tz);
}

__device__ double grad_noise2(double x, double y, uint32_t seed) {
  double fx = floor(x), fy = floor(y);
  int32_t ix = (int32_t)fx, iy = (int32_t)fy;
  double dx = x - fx, dy = y - fy;
  double v[4];
  for (int k = 0; k < 4; ++k) {
    int cx = k & 1, cy = k >> 1;
    uint32_t h = hash3(ix + cx, iy + cy, 0, seed);
    double ang = (h >> 8) * (6.283185307179586 / 16777216.0);
    v[k] = cos(ang) * (dx - cx) + sin(ang) * (dy - cy);
  }
  double tx = fade(dx), ty = fade(dy);
  return 1.4142135623730951 * lerp(lerp(v[0], v[1], tx), lerp(v[2], v[3], tx), ty);
}

__device__ double terrain_height(const Scene& s, double x, double y) {
  double h = 0.0, amp = 1.0, freq = 1.0 / s.terrain_scale, norm = 0.0;
  for (int o = 0; o < s.terrain_octaves; ++o) {
    h += amp * grad_noise2(x * freq, y * freq, s.terrain_seed + 977u * o);
    norm += amp;
    amp *= 0.5;
    freq *= 2.0;
  }
  return s.terrain_amp * h / norm;
}

__device__ double texture(const Scene& s, double x, double y, double z) {
  double v = 0.0, amp = 1.0, freq = s.tex_freq, norm = 0.0;
  for (int o = 0; o < s.tex_octaves; ++o) {
    v += amp * value_noise3(x * freq, y * freq, z * freq, s.tex_seed + 131u * o);
    norm += amp;
    amp *= 0.5;
    freq *= 2.0;
  }
  return v / norm;
}

__device__ double trace(const Scene& s, const double C[3], const double d[3], double nrm[3]) {
  double best = INFINITY;
  nrm[0] = 0; nrm[1] = 0; nrm[2] = 1;
  if (s.ground && !s.terrain && d[2] < 0.0) {
    double t = -C[2] / d[2];
    double gx = C[0] + t * d[0], gy = C[1] + t * d[1];
    int inside = s.ground_half <= 0.0 || (fabs(gx) <= s.ground_half && fabs(gy) <= s.ground_half);
    if (t > 0.0 && inside) best = t;
  }
  for (int b = 0; b < s.n_boxes; ++b) {
    const double* bx = s.boxes + 6 * b;
    double tn = -INFINITY, tf = INFINITY;
    int axis = -1, sign = 0, ok = 1;
    for (int a = 0; a < 3 && ok; ++a) {
      if (d[a] == 0.0) {
        if (C[a] < bx[a] || C[a] > bx[a + 3]) ok = 0;
        continue;
      }
      double t1 = (bx[a] - C[a]) / d[a], t2 = (bx[a + 3] - C[a]) / d[a];
      int s1 = -1;
      if (t1 > t2) { double tmp = t1; t1 = t2; t2 = tmp; s1 = 1; }
      if (t1 > tn) { tn = t1; axis = a; sign = s1; }
      if (t2 < tf) tf = t2;
    }
    if (!ok || tn > tf || tn <= 0.0 || axis < 0) continue;
    if (tn < best) {
      best = tn;
      nrm[0] = nrm[1] = nrm[2] = 0.0;
      nrm[axis] = (double)sign;
    }
  }
  if (s.terrain) {
    double tmax = best < 1e30 ? best : 2000.0;
    double step = 0.25, tprev = 0.0;
    double fprev = C[2] - terrain_height(s, C[0], C[1]);
    for (double t = step; t <= tmax; t += step) {
      double x = C[0] + t * d[0], y = C[1] + t * d[1], z = C[2] + t * d[2];
      double f = z - terrain_height(s, x, y);
      if (f <= 0.0 && fprev > 0.0) {
        double lo = tprev, hi = t;
        for (int it = 0; it < 40; ++it) {
          double mid = 0.5 * (lo + hi);
          double fm = C[2] + mid * d[2] - terrain_height(s, C[0] + mid * d[0], C[1] + mid * d[1]);
          if (fm > 0.0) lo = mid; else hi = mid;
        }
        double th = 0.5 * (lo + hi);
        if (th < best) {
          best = th;
          double x0 = C[0] + th * d[0], y0 = C[1] + th * d[1], e = 0.05;
          double gx = (terrain_height(s, x0 + e, y0) - terrain_height(s, x0 - e, y0)) / (2 * e);
          double gy = (terrain_height(s, x0, y0 + e) - terrain_height(s, x0, y0 - e)) / (2 * e);
          double n = sqrt(gx * gx + gy * gy + 1.0);
          nrm[0] = -gx / n; nrm[1] = -gy / n; nrm[2] = 1.0 / n;
        }
        break;
      }
      fprev = f;
      tprev = t;
      if (z < -10.0 * s.terrain_amp - 10.0 && d[2] < 0) break;
    }
  }
  return best;
}

__device__ double shade_sample(const Scene& s, const double C[3], const double d[3], double* tout) {
  double nrm[3];
  double t = trace(s, C, d, nrm);
  *tout = t;
  if (!(t < 1e30)) return -1.0;
  double X = C[0] + t * d[0], Y = C[1] + t * d[1], Z = C[2] + t * d[2];
  double tex = texture(s, X, Y, Z);
  const double L[3] = {0.4082482904638631, 0.4082482904638631, 0.8164965809277261};
  double lam = nrm[0] * L[0] + nrm[1] * L[1] + nrm[2] * L[2];
  if (lam < 0) lam = -lam * 0.5;
  return (0.5 + s.contrast * (tex - 0.5)) * (0.55 + 0.45 * lam);
}

// cams: per view K[9], R[9], t[3] (21 doubles).
__global__ void render_kernel(Scene s, const double* __restrict__ cams, int W, int H, int ss,
                              uint8_t* __restrict__ images, float* __restrict__ depths) {
  const int v = blockIdx.z;
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= H || j >= W) return;
  const double* K = cams + 21 * v;
  const double* R = K + 9;
  const double* tc = K + 18;
  double fx = K[0], skew = K[1], cx = K[2], fy = K[4], cy = K[5];
  double C[3];
  for (int a = 0; a < 3; ++a) C[a] = -(R[a] * tc[0] + R[3 + a] * tc[1] + R[6 + a] * tc[2]);
  double acc = 0.0;
  for (int sy = 0; sy < ss + 1; ++sy) {
    for (int sx = 0; sx < ss; ++sx) {
      double px, py;
      int centre = (sy == ss);
      if (centre) { if (sx) break; px = j; py = i; }
      else { px = j + (sx + 0.5) / ss - 0.5; py = i + (sy + 0.5) / ss - 0.5; }
      double yc = (py - cy) / fy;
      double xc = (px - cx - skew * yc) / fx;
      double dc[3] = {xc, yc, 1.0};
      double dw[3];
      for (int a = 0; a < 3; ++a) dw[a] = R[a] * dc[0] + R[3 + a] * dc[1] + R[6 + a] * dc[2];
      double t;
      double val = shade_sample(s, C, dw, &t);
      if (centre) {
        depths[((size_t)v * H + i) * W + j] = (t < 1e30) ? (float)t : 0.0f;
      } else {
        acc += (val >= 0.0) ? val : s.sky;
      }
    }
  }
  double val = acc / (ss * ss);
  double q = floor(255.0 * val + 0.5);
  if (q < 0) q = 0;
  if (q > 255) q = 255;
  images[((size_t)v * H + i) * W + j] = (uint8_t)q;
}

}  // namespace

// Renders n views of one scene into device buffers images [n][H][W] and
// depths [n][H][W]; cams is a device buffer of n x (K, R, t) doubles.
extern "C" int rcg_render(const double* boxes, int n_boxes, int ground, double ground_half,
                          int terrain, double terrain_amp, double terrain_scale,
                          uint32_t terrain_seed, int terrain_octaves, uint32_t tex_seed,
                          double tex_freq, int tex_octaves, double contrast, double sky,
                          const double* cams, int n_views, int W, int H, int ss, uint8_t* images,
                          float* depths, void* stream) {
  Scene s{boxes, n_boxes, ground, ground_half, terrain, terrain_amp, terrain_scale, terrain_seed,
          terrain_octaves, tex_seed, tex_freq, tex_octaves, contrast, sky};
  dim3 blk(32, 4), grid((W + 31) / 32, (H + 3) / 4, n_views);
  render_kernel<<<grid, blk, 0, static_cast<cudaStream_t>(stream)>>>(s, cams, W, H, ss, images,
                                                                      depths);
  return (int)cudaGetLastError();
}
