// Learned PatchMatch initialisation (no reference counterpart; the
// reference initialises at random, depthmap.cc:237-256).
//
//  - sweep_features_kernel: network input per pixel, NHWC BF16 with 32
//    channels: the reference intensity, then the bilateral NCC
//    (ComputePlaneImageScore) of 8 fronto-parallel planes uniform in inverse
//    depth against the 2 nearest matching views (16 channels), zeros after.
//  - conv3x3 forward / backward-data / backward-weight: 3x3 same-padding
//    convolutions over NHWC BF16 activations as implicit GEMMs on the tensor
//    cores (mma.sync m16n8k16, BF16 in, FP32 accumulate), bias and ReLU
//    fused in the epilogues.
//  - loss / Adam / plane kernels for training and for turning the network's
//    (inverse depth, normal slopes) into PatchMatch initial planes.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "learned.h"

namespace dn {

// ---------------------------------------------------------------- sweep
// L lanes per pixel, as the PatchMatch initialisation (the 7 x 7 patch).
// The features are computed on a grid of every S-th pixel in x and y
// (S = 1: every pixel): grid point (ys, xs) is the full-resolution pixel
// (S ys, S xs), scored with the full-resolution 7 x 7 patch around it.
// Blocks cover (blockDim.x / L) x blockDim.y grid points; the staged tile
// is the full-resolution region under them plus the patch halo.  Output:
// map k's grid point (ys, xs) at feat + base_k + (ys Ws + xs) 32, with
// base_k = k map_stride, or the map's proposal offset (MapDev::prop_off)
// times 32 when map_stride < 0.
template <int L, int S>
__global__ void __launch_bounds__(128)
sweep_features_kernel(const MapDev* __restrict__ maps, const ViewDev* __restrict__ views,
                      const PairDev* __restrict__ pairs, const int4* __restrict__ tiles,
                      __nv_bfloat16* __restrict__ feat, long long map_stride, int n_planes) {
  extern __shared__ float tile[];
  constexpr int HPZ = 3;
  const int4 tl = tiles[blockIdx.x];
  const MapDev& m = maps[tl.x];
  const ViewDev& rv = views[m.ref_view];
  const int W = m.W, H = m.H;
  const int Ws = (W + S - 1) / S, Hs = (H + S - 1) / S;
  const int px = blockDim.x / L;
  const int xs0 = tl.y * px, ys0 = tl.z * blockDim.y;
  const int x0 = S * xs0, y0 = S * ys0;
  const int pitch = S * px + 2 * HPZ, rows = S * blockDim.y + 2 * HPZ;
  __shared__ PairViewSm spv;
  for (int k = threadIdx.y * blockDim.x + threadIdx.x; k < pitch * rows;
       k += blockDim.x * blockDim.y) {
    const int r = k / pitch, c = k - r * pitch;
    const int y = min(max(y0 - HPZ + r, 0), H - 1), x = min(max(x0 - HPZ + c, 0), W - 1);
    tile[k] = __half2float(rv.img[(size_t)y * W + x]);
  }
  stage_pairs(spv, m, views, pairs);
  __syncthreads();
  const int g = threadIdx.x / L, lane = threadIdx.x % L;
  const unsigned mask = (L == 1) ? (1u << (threadIdx.x & 31))
                                 : (((1u << L) - 1u) << ((threadIdx.x & 31) & ~(L - 1)));
  const int ys = ys0 + threadIdx.y, xs = xs0 + g;
  // The lanes of a group share (ys, xs): a group leaves together.
  if (ys >= Hs || xs >= Ws) return;
  const int i = S * ys, j = S * xs;
  const int ly = S * threadIdx.y + HPZ, lx = S * g + HPZ;
  float f[kFeatC];
#pragma unroll
  for (int c = 0; c < kFeatC; ++c) f[c] = 0.f;
  f[0] = (tile[ly * pitch + lx] - 128.0f) * (1.0f / 64.0f);
  if (i >= HPZ && i < H - HPZ && j >= HPZ && j < W - HPZ) {
    Patch<HPZ, L> pt;
    pt.build(tile, pitch, ly, lx, lane, mask);
    const double a = 1.0 / m.min_depth, b = 1.0 / m.max_depth;
    unsigned taps = 0;
    const int nv = min(2, m.n_pairs);
    for (int p = 0; p < n_planes && p < kMaxSweepPlanes; ++p) {
      const float depth = (float)(1.0 / (a + (b - a) * (p + 0.5) / n_planes));
      const float3 v = plane_from_depth_normal((float)j, (float)i, m.Kinv_d, depth,
                                               make_float3(0.f, 0.f, -1.f));
      const Hyp h = make_hyp(m.Kinv, v, (float)j, (float)i);
      for (int k = 0; k < nv; ++k) {
        const PairDev& pr = spv.p[k];
        f[1 + 2 * p + k] = pt.view(spv.v[pr.view], pr, h, (float)j, (float)i, taps);
      }
    }
  }
  if (lane != 0) return;
  const long long base = map_stride >= 0 ? (long long)tl.x * map_stride : m.prop_off * kFeatC;
  __nv_bfloat16* out = feat + base + ((size_t)ys * Ws + xs) * kFeatC;
#pragma unroll
  for (int c = 0; c < kFeatC; c += 2)
    *reinterpret_cast<__nv_bfloat162*>(out + c) = __floats2bfloat162_rn(f[c], f[c + 1]);
}

// ------------------------------------------------------------ mma helper
__device__ inline void mma_bf16(float d[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ inline uint32_t ld_pair(const __nv_bfloat16* p) {
  return *reinterpret_cast<const uint32_t*>(p);
}
__device__ inline uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// Pixel index p of a batch of n images H x W -> (image, y, x); neighbour at
// offset (dy, dx) or -1 outside the image.
__device__ inline long long nbr_pixel(long long p, int H, int W, int dy, int dx) {
  const long long hw = (long long)H * W;
  const long long img = p / hw;
  const int r = (int)(p - img * hw);
  const int y = r / W + dy, x = r % W + dx;
  if (y < 0 || y >= H || x < 0 || x >= W) return -1;
  return img * hw + (long long)y * W + x;
}

// ------------------------------------------------------------ conv forward
// y[p][co] = b[co] + sum_{tap, ci} x[p + tap][ci] * w[co][tap * CIN + ci];
// M = pixels (16 per warp), N = COUT (padded to 8s), K = 9 * CIN.
// Weights ([COUT][9 CIN] BF16, k contiguous) are staged in shared memory.
template <int CIN, int COUT>
__global__ void __launch_bounds__(128)
conv3x3_fwd_kernel(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ w,
                   const float* __restrict__ bias, long long n_pix, int H, int W, int relu,
                   __nv_bfloat16* __restrict__ y, float* __restrict__ y32) {
  constexpr int K = 9 * CIN;
  constexpr int NT = (COUT + 7) / 8;
  __shared__ __align__(16) __nv_bfloat16 ws[NT * 8 * K];
  for (int k = threadIdx.x; k < NT * 8 * K; k += blockDim.x)
    ws[k] = (k / K) < COUT ? w[k] : __float2bfloat16(0.f);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const long long p0 = ((long long)blockIdx.x * 4 + warp) * 16;
  if (p0 >= n_pix) return;
  float acc[NT][4];
#pragma unroll
  for (int n = 0; n < NT; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
  const long long pa = p0 + g, pb = p0 + g + 8;
#pragma unroll 1
  for (int tap = 0; tap < 9; ++tap) {
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    const long long qa = pa < n_pix ? nbr_pixel(pa, H, W, dy, dx) : -1;
    const long long qb = pb < n_pix ? nbr_pixel(pb, H, W, dy, dx) : -1;
#pragma unroll
    for (int c0 = 0; c0 < CIN; c0 += 16) {
      const uint32_t a0 = qa >= 0 ? ld_pair(x + qa * CIN + c0 + 2 * t) : 0u;
      const uint32_t a1 = qb >= 0 ? ld_pair(x + qb * CIN + c0 + 2 * t) : 0u;
      const uint32_t a2 = qa >= 0 ? ld_pair(x + qa * CIN + c0 + 2 * t + 8) : 0u;
      const uint32_t a3 = qb >= 0 ? ld_pair(x + qb * CIN + c0 + 2 * t + 8) : 0u;
      const int kk = tap * CIN + c0 + 2 * t;
#pragma unroll
      for (int n = 0; n < NT; ++n) {
        const __nv_bfloat16* wr = ws + (n * 8 + g) * K + kk;
        mma_bf16(acc[n], a0, a1, a2, a3, ld_pair(wr), ld_pair(wr + 8));
      }
    }
  }
#pragma unroll
  for (int n = 0; n < NT; ++n) {
    const int co = n * 8 + 2 * t;
    if (co >= COUT) continue;
    const float b0 = bias[co], b1 = (co + 1 < COUT) ? bias[co + 1] : 0.f;
    float v[4] = {acc[n][0] + b0, acc[n][1] + b1, acc[n][2] + b0, acc[n][3] + b1};
    if (relu)
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] = fmaxf(v[k], 0.f);
    const long long rows[2] = {pa, pb};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long p = rows[h];
      if (p >= n_pix) continue;
      if (y) {
        if (co + 1 < COUT)
          *reinterpret_cast<__nv_bfloat162*>(y + p * COUT + co) =
              __floats2bfloat162_rn(v[2 * h], v[2 * h + 1]);
        else
          y[p * COUT + co] = __float2bfloat16(v[2 * h]);
      }
      if (y32) {
        y32[p * COUT + co] = v[2 * h];
        if (co + 1 < COUT) y32[p * COUT + co + 1] = v[2 * h + 1];
      }
    }
  }
}

// ------------------------------------------------ conv forward, tcgen05
// The same convolution on the 5th-generation tensor cores.  A CTA of 4
// warps computes a spatial tile of 16 rows x 8 columns of one image (128
// pixels, the GEMM's M) for N = the output channels (32, or 16 holding the
// 4 outputs of the last layer), K = 9 taps x 32 input channels in 18 MMAs
// of K = 16.  The tile's input with a one-pixel halo (18 x 10 pixels x 32
// channels, 11.5 KB) is copied once into shared memory, as four planes of
// 8 channels, 16 bytes per pixel: for tap (dy, dx) the A operand of the
// tile is then a strided view of that buffer in the canonical no-swizzle
// K-major layout -- 8-pixel core-matrix rows of 16 bytes, 8-row groups one
// halo row (160 bytes) apart (SBO), the two 8-channel halves of one MMA's
// K one plane (2880 bytes) apart (LBO) -- so no im2col copy is made.  The
// weights (B, [cout][9 x 32]) are staged once per CTA in the same layout
// (8-row groups 128 bytes apart).  Thread 0 issues the MMAs into a 128 x N
// FP32 accumulator in tensor memory and commits them to an mbarrier; the
// halo of the CTA's next tile streams in with cp.async meanwhile (two
// buffers).  Every warp then reads its 32 accumulator lanes (its 32
// pixels) with tcgen05.ld, adds the bias, applies the ReLU and stores.
// Each wait is bounded and sets an error word on expiry.
namespace tc {

__device__ int g_error;

constexpr int kTR = 16, kTC = 8;             // tile rows x columns (M = 128)
constexpr int kHR = kTR + 2, kHC = kTC + 2;  // halo buffer rows x columns
constexpr int kPlane = kHR * kHC * 16;       // bytes of one 8-channel plane
constexpr int kHalo = 4 * kPlane;            // 32 channels
constexpr int kK = 9 * 32;                   // GEMM K
constexpr int kKC = kK / 8;                  // 16-byte K chunks of the weights
constexpr long long kSpins = 1LL << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, K-major without swizzle: start address,
// leading-dimension byte offset (between the K halves), stride-dimension
// byte offset (between 8-row groups), all in 16-byte units; bit 46 is the
// sm_100 descriptor version.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1),
// A and B BF16 (bits 7-9, 10-12 = 1), both K-major, N / 8 at bit 17,
// M / 16 = 8 at bit 24.
constexpr uint32_t idesc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | (8u << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t phase) {
  for (long long i = 0; i < kSpins; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16-byte asynchronous copy; src_bytes = 0 writes zeros (outside the image).
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
               "r"(src_bytes)
               : "memory");
}

template <int NP>
__device__ __forceinline__ void tmem_load(uint32_t taddr, uint32_t (&r)[NP]);

template <>
__device__ __forceinline__ void tmem_load<32>(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

template <>
__device__ __forceinline__ void tmem_load<16>(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

constexpr size_t smem_bytes(int np) { return 2 * (size_t)kHalo + (size_t)kKC * np * 16 + 32; }

// Tile t of the batch: image, first row, first column.
struct TileXY {
  long long img;
  int y0, x0;
};
__device__ __forceinline__ TileXY tile_xy(long long t, int H, int W) {
  const int ty = (H + kTR - 1) / kTR, tx = (W + kTC - 1) / kTC;
  const long long per = (long long)ty * tx;
  TileXY r;
  r.img = t / per;
  const int k = (int)(t - r.img * per);
  r.y0 = (k / tx) * kTR;
  r.x0 = (k % tx) * kTC;
  return r;
}

// Issues the copies of tile t's halo into `buf` (one commit group).
__device__ __forceinline__ void load_halo(uint32_t buf, const __nv_bfloat16* x, long long t, int H,
                                          int W) {
  const TileXY tt = tile_xy(t, H, W);
  for (int e = threadIdx.x; e < kHR * kHC * 4; e += blockDim.x) {
    const int hp = e >> 2, j = e & 3;
    const int y = tt.y0 - 1 + hp / kHC, xx = tt.x0 - 1 + hp % kHC;
    const bool in = y >= 0 && y < H && xx >= 0 && xx < W;
    const long long q = in ? (tt.img * H + y) * (long long)W + xx : 0;
    cp_async16(buf + (uint32_t)(j * kPlane + hp * 16), x + q * 32 + j * 8, in ? 16u : 0u);
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

}  // namespace tc

template <int NP>
__global__ void __launch_bounds__(128, 4)
conv3x3_fwd_tc_kernel(const __nv_bfloat16* __restrict__ x, const __nv_bfloat16* __restrict__ w,
                      const float* __restrict__ bias, int H, int W, int cout, int relu,
                      __nv_bfloat16* __restrict__ y, float* __restrict__ y32, long long n_tiles,
                      const __nv_bfloat16* __restrict__ mask) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* halo = smem;                    // 2 x [4 planes][kHR][kHC][16 B]
  unsigned char* Bs = smem + 2 * kHalo;          // [kKC][NP][16 B]
  uint64_t* mbar = reinterpret_cast<uint64_t*>(Bs + (size_t)kKC * NP * 16);  // 2 barriers
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 2);
  const int tid = threadIdx.x, warp = tid >> 5;
  constexpr uint32_t kCols = 2 * NP;  // two accumulators (32 or 64 columns)

  long long t = blockIdx.x;
  const uint32_t h_base = smem_u32(halo);
  if (t < n_tiles) load_halo(h_base, x, t, H, W);
  for (int e = tid; e < kKC * NP; e += blockDim.x) {
    const int kc = e / NP, n = e - kc * NP;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (n < cout) v = *reinterpret_cast<const uint4*>(w + (size_t)n * kK + kc * 8);
    *reinterpret_cast<uint4*>(Bs + (size_t)e * 16) = v;
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(mbar + 1)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(tslot)), "n"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t b_base = smem_u32(Bs), mb0 = smem_u32(mbar);
  constexpr uint32_t idesc = idesc_bf16(NP);
  const long long G = gridDim.x;
  // Tile k of this CTA (t = blockIdx.x + k G) uses halo buffer and
  // accumulator k & 1.  The MMAs of tile k + 1 are issued before the
  // epilogue of tile k, and the halo of tile k + 2 streams in meanwhile.
  auto issue = [&](int buf) {
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a_base = h_base + (uint32_t)(buf * kHalo);
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint32_t a_off = (uint32_t)(2 * h * kPlane + ((tap / 3) * kHC + tap % 3) * 16);
          const uint64_t ad = smem_desc(a_base + a_off, kPlane, kHC * 16);
          const uint64_t bd =
              smem_desc(b_base + (uint32_t)((tap * 4 + 2 * h) * NP * 16), NP * 16, 128);
          const uint32_t acc = (tap | h) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
                  tmem + (uint32_t)(buf * NP)),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
              : "memory");
        }
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
              mb0 + 8u * (uint32_t)buf)
          : "memory");
    }
  };
  // The generic-proxy and cp.async writes of the halo become visible to
  // the tensor core; the previous readers of the accumulator are done.
  auto halo_ready = [&]() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
  };
  uint32_t phase[2] = {0u, 0u};
  int pend = -1;  // accumulator whose MMAs are in flight and not yet waited for
  int cur = 0;
  bool ok = true;
  if (t < n_tiles) {
    halo_ready();
    issue(0);
    pend = 0;
    if (t + G < n_tiles) load_halo(h_base + (uint32_t)kHalo, x, t + G, H, W);
  }
  for (; t < n_tiles; t += G) {
    const long long tn = t + G;
    if (tn < n_tiles) {
      halo_ready();
      issue(cur ^ 1);
    }
    bool done = mbar_wait(mb0 + 8u * (uint32_t)cur, phase[cur]);
    if (!done) done = mbar_wait(mb0 + 8u * (uint32_t)cur, phase[cur]);  // a late completion
    phase[cur] ^= 1u;
    pend = tn < n_tiles ? (cur ^ 1) : -1;
    ok = __syncthreads_and(done) != 0;
    if (!ok) break;
    // Tile k's halo buffer is free: the halo of tile k + 2 streams into it.
    if (tn + G < n_tiles) load_halo(h_base + (uint32_t)(cur * kHalo), x, tn + G, H, W);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    uint32_t r[NP];
    tmem_load<NP>(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cur * NP), r);
    const TileXY tt = tile_xy(t, H, W);
    const int py = tt.y0 + (tid >> 3), px = tt.x0 + (tid & 7);
    if (py < H && px < W) {
      const long long p = (tt.img * H + py) * (long long)W + px;
      if (NP == 32) {
        uint32_t o[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          float v0 = __uint_as_float(r[2 * c]) + (bias ? bias[2 * c] : 0.f);
          float v1 = __uint_as_float(r[2 * c + 1]) + (bias ? bias[2 * c + 1] : 0.f);
          if (relu) {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
          }
          if (mask) {
            // The gradient of a ReLU input: zero where the activation is not
            // positive (backward-data through the layer below's ReLU).
            const __nv_bfloat162 mk = *reinterpret_cast<const __nv_bfloat162*>(mask + p * 32 + 2 * c);
            if (!(__low2float(mk) > 0.f)) v0 = 0.f;
            if (!(__high2float(mk) > 0.f)) v1 = 0.f;
          }
          o[c] = pack2(__float2bfloat16_rn(v0), __float2bfloat16_rn(v1));
        }
        if (y) {
          uint4* dst = reinterpret_cast<uint4*>(y + p * 32);
#pragma unroll
          for (int j = 0; j < 4; ++j)
            dst[j] = make_uint4(o[4 * j], o[4 * j + 1], o[4 * j + 2], o[4 * j + 3]);
        }
        if (y32)
#pragma unroll
          for (int c = 0; c < 32; ++c) {
            const float v = __uint_as_float(r[c]) + (bias ? bias[c] : 0.f);
            y32[p * 32 + c] = relu ? fmaxf(v, 0.f) : v;
          }
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (c >= cout) break;
          float v = __uint_as_float(r[c]) + (bias ? bias[c] : 0.f);
          if (relu) v = fmaxf(v, 0.f);
          if (y) y[p * cout + c] = __float2bfloat16_rn(v);
          if (y32) y32[p * cout + c] = v;
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    cur ^= 1;
  }
  if (!ok && pend >= 0) {
    // A wait ran out: wait (bounded) for the MMAs still in flight before the
    // accumulators are freed.
    mbar_wait(mb0 + 8u * (uint32_t)pend, phase[pend]);
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  if (!ok && tid == 0) atomicExch(&g_error, 1);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "n"(kCols)
                 : "memory");
}

// ------------------------------------------------------- conv backward-data
// dx[p][ci] = mask(x_in[p][ci] > 0) * sum_{tap, co} dy[p - tap][co] *
// wt[ci][tap * COUT + co], wt the weights transposed to [CIN][9 COUT].
template <int CIN, int COUT>
__global__ void __launch_bounds__(128)
conv3x3_bwd_data_kernel(const __nv_bfloat16* __restrict__ dy, const __nv_bfloat16* __restrict__ wt,
                        const __nv_bfloat16* __restrict__ x_in, long long n_pix, int H, int W,
                        __nv_bfloat16* __restrict__ dx) {
  constexpr int COUTP = ((COUT + 15) / 16) * 16;  // K chunks of 16
  constexpr int K = 9 * COUTP;
  constexpr int NT = CIN / 8;
  __shared__ __align__(16) __nv_bfloat16 ws[CIN * K];
  for (int k = threadIdx.x; k < CIN * K; k += blockDim.x) ws[k] = wt[k];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const long long p0 = ((long long)blockIdx.x * 4 + warp) * 16;
  if (p0 >= n_pix) return;
  float acc[NT][4];
#pragma unroll
  for (int n = 0; n < NT; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
  const long long pa = p0 + g, pb = p0 + g + 8;
#pragma unroll 1
  for (int tap = 0; tap < 9; ++tap) {
    const int dyy = 1 - tap / 3, dxx = 1 - tap % 3;  // dy at p - (tap offset)
    const long long qa = pa < n_pix ? nbr_pixel(pa, H, W, dyy, dxx) : -1;
    const long long qb = pb < n_pix ? nbr_pixel(pb, H, W, dyy, dxx) : -1;
#pragma unroll
    for (int c0 = 0; c0 < COUTP; c0 += 16) {
      auto ld = [&](long long q, int c) -> uint32_t {
        if (q < 0) return 0u;
        const __nv_bfloat16 lo = c < COUT ? dy[q * COUT + c] : __float2bfloat16(0.f);
        const __nv_bfloat16 hi = c + 1 < COUT ? dy[q * COUT + c + 1] : __float2bfloat16(0.f);
        return pack2(lo, hi);
      };
      const uint32_t a0 = ld(qa, c0 + 2 * t), a1 = ld(qb, c0 + 2 * t);
      const uint32_t a2 = ld(qa, c0 + 2 * t + 8), a3 = ld(qb, c0 + 2 * t + 8);
      const int kk = tap * COUTP + c0 + 2 * t;
#pragma unroll
      for (int n = 0; n < NT; ++n) {
        const __nv_bfloat16* wr = ws + (n * 8 + g) * K + kk;
        mma_bf16(acc[n], a0, a1, a2, a3, ld_pair(wr), ld_pair(wr + 8));
      }
    }
  }
#pragma unroll
  for (int n = 0; n < NT; ++n) {
    const int ci = n * 8 + 2 * t;
    const long long rows[2] = {pa, pb};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const long long p = rows[h];
      if (p >= n_pix) continue;
      float v0 = acc[n][2 * h], v1 = acc[n][2 * h + 1];
      if (x_in) {
        const __nv_bfloat162 xi = *reinterpret_cast<const __nv_bfloat162*>(x_in + p * CIN + ci);
        if (!(__low2float(xi) > 0.f)) v0 = 0.f;
        if (!(__high2float(xi) > 0.f)) v1 = 0.f;
      }
      *reinterpret_cast<__nv_bfloat162*>(dx + p * CIN + ci) = __floats2bfloat162_rn(v0, v1);
    }
  }
}

// Weights [COUT][9 CIN] -> [CIN][9 COUTP] (COUTP = COUT padded to 16).
__global__ void transpose_weights_kernel(const __nv_bfloat16* __restrict__ w, int cin, int cout,
                                         int coutp, __nv_bfloat16* __restrict__ wt) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = cin * 9 * coutp;
  if (k >= n) return;
  const int ci = k / (9 * coutp), r = k - ci * 9 * coutp, tap = r / coutp, co = r - tap * coutp;
  wt[k] = co < cout ? w[(size_t)co * 9 * cin + tap * cin + ci] : __float2bfloat16(0.f);
}

// ------------------------------------------ conv backward-weight, tcgen05
// dw[co][tap * 32 + ci] += sum_p g[p][co] x[p + off(tap)][ci] and
// db[co] += sum_p g[p][co], off(tap) = (tap / 3 - 1, tap % 3 - 1), as a
// split-K GEMM on the tensor cores.  A CTA walks tiles of 16 x 8 pixels
// (K = 128 per tile) and keeps three 128 x N FP32 accumulators in tensor
// memory, one per vertical offset dy = d - 1:
//   D_d[m = (dxs, ci)][n = co] += sum_k A_d[m][k] B[n][k],
//   A_d[(dxs, ci)][(r, c)] = x[y0 + r + d - 1][x0 + c + dxs - 1][ci] (dxs < 3),
//   B[co][(r, c)] = g[y0 + r][x0 + c][co],
// so D_d row (dxs, ci), column co is dw[co][(3 d + dxs) * 32 + ci].  Row
// block dxs = 3 of A stays zero (M = 128 = 4 x 32).  Operands are staged in
// shared memory in the canonical no-swizzle K-major layout (a core matrix is
// 8 rows of 8 K-elements, 16 bytes a row, 128 contiguous bytes):
//   A: halo row hr (18 rows) x [dxs 4][ci 32][8 px]: 8-row groups 128 B
//      apart (SBO), the two K-halves of an MMA (tile rows 2c and 2c + 1)
//      one halo row (2048 B) apart (LBO); A_d of K-chunk c starts at halo
//      row 2c + d;
//   B: tile row r (16) x [co N][8 px]: SBO 128 B, LBO N x 16 B.
// x is NHWC BF16 with 32 channels, g NHWC BF16 with ldg channels per pixel
// of which the first cout are used.  Two operand buffers: the loads of tile
// t + 1 overlap the MMAs of tile t.  Each CTA adds its sums to dw and db
// once, at the end, with atomics.  Waits are bounded (tc::kSpins); an
// expired wait sets tc::g_error and the CTA stops.
namespace tcw {
constexpr int kTR = 16, kTC = 8, kHR = kTR + 2;
constexpr int kARow = 4 * 32 * 16;    // one halo row of A: 2048 bytes
constexpr int kABytes = kHR * kARow;  // 36864 bytes
__host__ __device__ constexpr int b_row(int n) { return n * 16; }
__host__ __device__ constexpr int buf_bytes(int n) { return kABytes + kTR * b_row(n); }
constexpr size_t smem_bytes(int n) { return 2 * (size_t)buf_bytes(n) + 64; }
}  // namespace tcw

template <int N>
__global__ void __launch_bounds__(128, 2)
conv3x3_bwd_weight_tc_kernel(const __nv_bfloat16* __restrict__ g, int ldg, int cout,
                             const __nv_bfloat16* __restrict__ x, int H, int W,
                             long long n_tiles, float* __restrict__ dw, float* __restrict__ db) {
  using namespace tc;
  static_assert(N == 16 || N == 32, "N: output channels padded to 16 or 32");
  static_assert(tcw::kTR == tc::kTR && tcw::kTC == tc::kTC, "the forward's tiling");
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + 2 * tcw::buf_bytes(N));
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int e = tid; e < 2 * tcw::buf_bytes(N) / 16; e += blockDim.x)
    reinterpret_cast<uint4*>(smem)[e] = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(mbar)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(mbar + 1)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;\n" ::"r"(
                     smem_u32(tslot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  // db: the B loads of thread tid always carry channel tid % N (the block's
  // 128 threads are a multiple of N), so each thread sums one channel.
  float bsum = 0.f;

  auto load_tile = [&](long long t, int b) {
    unsigned char* A = smem + b * tcw::buf_bytes(N);
    unsigned char* Bm = A + tcw::kABytes;
    const TileXY tt = tile_xy(t, H, W);
    for (int e = tid; e < tcw::kHR * 3 * 32; e += blockDim.x) {
      const int ci = e & 31, q = e >> 5, dxs = q % 3, hr = q / 3;
      const int y = tt.y0 - 1 + hr;
      uint32_t pk[4];
#pragma unroll
      for (int c2 = 0; c2 < 4; ++c2) {
        __nv_bfloat16 v[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int xx = tt.x0 + 2 * c2 + h + dxs - 1;
          const bool in = y >= 0 && y < H && xx >= 0 && xx < W;
          v[h] = in ? x[((tt.img * H + y) * (long long)W + xx) * 32 + ci] : __float2bfloat16(0.f);
        }
        pk[c2] = pack2(v[0], v[1]);
      }
      *reinterpret_cast<uint4*>(A + hr * tcw::kARow + (dxs * 32 + ci) * 16) =
          make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
    for (int e = tid; e < tcw::kTR * N; e += blockDim.x) {
      const int co = e % N, r = e / N;
      const int y = tt.y0 + r;
      uint32_t pk[4];
#pragma unroll
      for (int c2 = 0; c2 < 4; ++c2) {
        __nv_bfloat16 v[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int xx = tt.x0 + 2 * c2 + h;
          const bool in = co < cout && y < H && xx < W;
          v[h] = in ? g[((tt.img * H + y) * (long long)W + xx) * ldg + co] : __float2bfloat16(0.f);
          bsum += __bfloat162float(v[h]);
        }
        pk[c2] = pack2(v[0], v[1]);
      }
      *reinterpret_cast<uint4*>(Bm + r * tcw::b_row(N) + co * 16) =
          make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
  };

  constexpr uint32_t idesc = idesc_bf16(N);
  uint32_t phase[2] = {0u, 0u};
  bool pending[2] = {false, false};
  bool ok = true, first = true;
  int buf = 0;
  long long t = blockIdx.x;
  if (t < n_tiles) load_tile(t, 0);
  for (; t < n_tiles && ok; t += gridDim.x) {
    // The generic-proxy stores of this buffer become visible to the tensor
    // core; then one thread issues the tile's 24 MMAs.
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t a_base = smem_u32(smem + buf * tcw::buf_bytes(N));
      const uint32_t b_base = a_base + tcw::kABytes;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const uint64_t bd =
            smem_desc(b_base + (uint32_t)(2 * c * tcw::b_row(N)), tcw::b_row(N), 128);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const uint64_t ad =
              smem_desc(a_base + (uint32_t)((2 * c + d) * tcw::kARow), tcw::kARow, 128);
          const uint32_t acc = (first && c == 0) ? 0u : 1u;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
                  tmem + (uint32_t)(d * N)),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
              : "memory");
        }
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
              smem_u32(mbar + buf))
          : "memory");
    }
    pending[buf] = true;
    first = false;
    const long long tn = t + gridDim.x;
    const int nb = buf ^ 1;
    if (tn < n_tiles) {
      if (pending[nb]) {
        // The MMAs that last read buffer nb must be done before it is reused.
        bool done = mbar_wait(smem_u32(mbar + nb), phase[nb]);
        if (!done) done = mbar_wait(smem_u32(mbar + nb), phase[nb]);
        phase[nb] ^= 1u;
        pending[nb] = false;
        ok = __syncthreads_and(done) != 0;
        if (!ok) break;
      }
      load_tile(tn, nb);
    }
    buf = nb;
  }
  for (int b = 0; b < 2; ++b) {
    if (!pending[b]) continue;
    bool done = mbar_wait(smem_u32(mbar + b), phase[b]);
    if (!done) done = mbar_wait(smem_u32(mbar + b), phase[b]);
    ok = ok && done;
  }
  ok = __syncthreads_and(ok) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (ok && !first) {
    if (warp < 3) {  // warp 3's TMEM lanes hold the zero row block
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        uint32_t r[N];
        tmem_load<N>(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(d * N), r);
        const int tap = 3 * d + warp, ci = lane;
#pragma unroll
        for (int co = 0; co < N; ++co)
          if (co < cout) atomicAdd(dw + (size_t)co * 288 + tap * 32 + ci, __uint_as_float(r[co]));
      }
    }
    const int co = tid % N;
    if (co < cout && bsum != 0.f) atomicAdd(db + co, bsum);
  }
  if (!ok && tid == 0) atomicExch(&g_error, 1);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;\n" ::"r"(tmem) : "memory");
}

// Backward-data weights for the forward tcgen05 kernel: the gradient of a
// layer's input is conv3x3(g, w') with w'[ci][tap * 32 + co] =
// w[co][(8 - tap) * 32 + ci] (taps flipped, channels swapped) for co < cout,
// zero for co >= cout (g padded to 32 channels).
__global__ void flip_weights_kernel(const __nv_bfloat16* __restrict__ w, int cout,
                                    __nv_bfloat16* __restrict__ wf) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 32 * 288) return;
  const int ci = k / 288, r = k - ci * 288, tap = r / 32, co = r - tap * 32;
  wf[k] = co < cout ? w[(size_t)co * 288 + (8 - tap) * 32 + ci] : __float2bfloat16(0.f);
}

// [n][cin] -> [n][32] with zeros after channel cin.
__global__ void pad_channels_kernel(const __nv_bfloat16* __restrict__ src, int cin, long long n,
                                    __nv_bfloat16* __restrict__ dst) {
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= n * 32) return;
  const long long p = k >> 5;
  const int c = (int)(k & 31);
  dst[k] = c < cin ? src[p * cin + c] : __float2bfloat16(0.f);
}

// ----------------------------------------------------- conv backward-weight
// dw[co][tap * CIN + ci] += sum_p dy[p][co] * x[p + tap][ci]: M = COUT
// (tiles of 16), N = 9 CIN (tiles of 8, split over the 4 warps), K = pixels.
// Each block reduces a chunk of pixels and adds its partial sums atomically.
template <int CIN, int COUT>
__global__ void __launch_bounds__(128)
conv3x3_bwd_weight_kernel(const __nv_bfloat16* __restrict__ dy, const __nv_bfloat16* __restrict__ x,
                          long long n_pix, int H, int W, int pix_per_block,
                          float* __restrict__ dw, float* __restrict__ db) {
  constexpr int MT = (COUT + 15) / 16;
  constexpr int NTOT = 9 * CIN / 8;
  constexpr int NW = (NTOT + 3) / 4;  // n tiles per warp
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  float acc[MT][NW][4];
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int n = 0; n < NW; ++n) acc[m][n][0] = acc[m][n][1] = acc[m][n][2] = acc[m][n][3] = 0.f;
  float bsum[2] = {0.f, 0.f};
  const long long pbeg = (long long)blockIdx.x * pix_per_block;
  const long long pend = min(pbeg + pix_per_block, n_pix);
  auto dyv = [&](long long p, int co) -> __nv_bfloat16 {
    return (p < pend && co < COUT) ? dy[p * COUT + co] : __float2bfloat16(0.f);
  };
#pragma unroll 1
  for (long long pk = pbeg; pk < pend; pk += 16) {
    // A fragments: rows co, k = pixels pk + 2t (+1, +8, +9).
    uint32_t a[MT][4];
#pragma unroll
    for (int m = 0; m < MT; ++m) {
      const int ca = m * 16 + g, cb = ca + 8;
      a[m][0] = pack2(dyv(pk + 2 * t, ca), dyv(pk + 2 * t + 1, ca));
      a[m][1] = pack2(dyv(pk + 2 * t, cb), dyv(pk + 2 * t + 1, cb));
      a[m][2] = pack2(dyv(pk + 2 * t + 8, ca), dyv(pk + 2 * t + 9, ca));
      a[m][3] = pack2(dyv(pk + 2 * t + 8, cb), dyv(pk + 2 * t + 9, cb));
    }
    if (warp == 0) {
      // Bias gradient: lanes 0..15 own output channel 2 lanes each... simple
      // per-lane sums over this 16-pixel step for co = lane, lane + 32.
      for (int c = lane; c < COUT; c += 32)
        for (int q = 0; q < 16; ++q) bsum[c / 32] += __bfloat162float(dyv(pk + q, c));
    }
#pragma unroll
    for (int n = 0; n < NW; ++n) {
      const int nt = warp * NW + n;
      if (nt >= NTOT) break;
      const int col = nt * 8 + g;  // (tap, ci)
      const int tap = col / CIN, ci = col - tap * CIN;
      const int dyy = tap / 3 - 1, dxx = tap % 3 - 1;
      auto xv = [&](long long p) -> __nv_bfloat16 {
        if (p >= pend) return __float2bfloat16(0.f);
        const long long q = nbr_pixel(p, H, W, dyy, dxx);
        return q >= 0 ? x[q * CIN + ci] : __float2bfloat16(0.f);
      };
      const uint32_t b0 = pack2(xv(pk + 2 * t), xv(pk + 2 * t + 1));
      const uint32_t b1 = pack2(xv(pk + 2 * t + 8), xv(pk + 2 * t + 9));
#pragma unroll
      for (int m = 0; m < MT; ++m) mma_bf16(acc[m][n], a[m][0], a[m][1], a[m][2], a[m][3], b0, b1);
    }
  }
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int n = 0; n < NW; ++n) {
      const int nt = warp * NW + n;
      if (nt >= NTOT) break;
      const int co_a = m * 16 + g, co_b = co_a + 8, col = nt * 8 + 2 * t;
      if (co_a < COUT) {
        atomicAdd(dw + (size_t)co_a * 9 * CIN + col, acc[m][n][0]);
        atomicAdd(dw + (size_t)co_a * 9 * CIN + col + 1, acc[m][n][1]);
      }
      if (co_b < COUT) {
        atomicAdd(dw + (size_t)co_b * 9 * CIN + col, acc[m][n][2]);
        atomicAdd(dw + (size_t)co_b * 9 * CIN + col + 1, acc[m][n][3]);
      }
    }
  if (warp == 0)
    for (int c = lane; c < COUT; c += 32) atomicAdd(db + c, bsum[c / 32]);
}

// ------------------------------------------------------------- loss / Adam
// Output channels: 0 inverse depth t in [0, 1] over the depth range,
// 1-2 normal slopes (sx, sy), normal ~ (sx, sy, -1).  L1 loss on pixels with
// target weight > 0; gradient written as BF16 for the last layer's backward.
__global__ void l1_loss_kernel(const float* __restrict__ pred, const float* __restrict__ target,
                               long long n_pix, float normal_weight, __nv_bfloat16* __restrict__ dpred,
                               float* __restrict__ loss_sum, float* __restrict__ count) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  float l = 0.f, c = 0.f;
  if (p < n_pix) {
    const float4 tg = *reinterpret_cast<const float4*>(target + 4 * p);  // t, sx, sy, weight
    const float wgt = tg.w;
    float g[4] = {0.f, 0.f, 0.f, 0.f};
    if (wgt > 0.f) {
      const float d0 = pred[4 * p] - tg.x, d1 = pred[4 * p + 1] - tg.y, d2 = pred[4 * p + 2] - tg.z;
      l = wgt * (fabsf(d0) + normal_weight * (fabsf(d1) + fabsf(d2)));
      c = wgt;
      g[0] = wgt * copysignf(1.f, d0);
      g[1] = wgt * normal_weight * copysignf(1.f, d1);
      g[2] = wgt * normal_weight * copysignf(1.f, d2);
    }
    *reinterpret_cast<__nv_bfloat162*>(dpred + 4 * p) = __floats2bfloat162_rn(g[0], g[1]);
    *reinterpret_cast<__nv_bfloat162*>(dpred + 4 * p + 2) = __floats2bfloat162_rn(g[2], g[3]);
  }
  for (int o = 16; o; o >>= 1) {
    l += __shfl_xor_sync(0xffffffffu, l, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(loss_sum, l);
    atomicAdd(count, c);
  }
}

// Adam on FP32 master weights (grad scaled by 1 / count), BF16 copy out.
__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ grad, int n, const float* __restrict__ count,
                            float lr, float b1, float b2, float eps, float bc1, float bc2,
                            __nv_bfloat16* __restrict__ w16) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float c = fmaxf(*count, 1.f);
  const float gr = grad[k] / c;
  const float mk = b1 * m[k] + (1.f - b1) * gr;
  const float vk = b2 * v[k] + (1.f - b2) * gr * gr;
  m[k] = mk;
  v[k] = vk;
  const float nw = w[k] - lr * (mk / bc1) / (sqrtf(vk / bc2) + eps);
  w[k] = nw;
  if (w16) w16[k] = __float2bfloat16(nw);
}

// Network output -> PatchMatch initial planes for one map: depth from the
// inverse-depth fraction, normal (sx, sy, -1), plane through the back-
// projected point (PlaneFromDepthAndNormal, depthmap.cc:120-125).
__global__ void output_to_planes_kernel(const float* __restrict__ out, int W, int H,
                                        const MapDev* __restrict__ maps, int map,
                                        float* __restrict__ planes) {
  const MapDev& m = maps[map];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= W * H) return;
  const int i = k / W, j = k - i * W;
  const float t = fminf(fmaxf(out[4 * k], 0.f), 1.f);
  const double a = 1.0 / m.max_depth, b = 1.0 / m.min_depth;
  const float depth = (float)(1.0 / (a + (b - a) * (double)t));
  const float sx = fminf(fmaxf(out[4 * k + 1], -4.f), 4.f);
  const float sy = fminf(fmaxf(out[4 * k + 2], -4.f), 4.f);
  const float3 v = plane_from_depth_normal((float)j, (float)i, m.Kinv_d, depth,
                                           make_float3(sx, sy, -1.f));
  planes[3 * (size_t)k] = v.x;
  planes[3 * (size_t)k + 1] = v.y;
  planes[3 * (size_t)k + 2] = v.z;
}

// Proposal grid output -> initial planes of every map of the batch
// (blockIdx.y = map): the network's (t, sx, sy) at full-resolution pixel
// (i, j) are the bilinear interpolation of the grid values around
// (i / S, j / S) (grid point (ys, xs) sits on pixel (S ys, S xs); clamped
// at the grid's last row and column), S the map's grid stride
// (MapDev::prop_S), then the same depth and plane as
// output_to_planes_kernel.  Writes MapDev::prop_init.
__global__ void proposal_to_planes_kernel(const float* __restrict__ out,
                                          const MapDev* __restrict__ maps) {
  const MapDev& m = maps[blockIdx.y];
  const int W = m.W, H = m.H, S = m.prop_S;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= W * H) return;
  const int i = k / W, j = k - i * W;
  const int Ws = m.prop_W, Hs = m.prop_H;
  const float* o = out + 4 * m.prop_off;
  float t, sx, sy;
  if (S == 1) {
    t = o[4 * (size_t)k];
    sx = o[4 * (size_t)k + 1];
    sy = o[4 * (size_t)k + 2];
  } else {
    const int y0 = min(i / S, Hs - 1), x0 = min(j / S, Ws - 1);
    const int y1 = min(y0 + 1, Hs - 1), x1 = min(x0 + 1, Ws - 1);
    const float inv = 1.0f / (float)S;  // exact: S is a power of two
    const float fy = (float)(i - S * y0) * inv, fx = (float)(j - S * x0) * inv;
    const float* q00 = o + 4 * ((size_t)y0 * Ws + x0);
    const float* q01 = o + 4 * ((size_t)y0 * Ws + x1);
    const float* q10 = o + 4 * ((size_t)y1 * Ws + x0);
    const float* q11 = o + 4 * ((size_t)y1 * Ws + x1);
    float v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float top = fmaf(fx, q01[c] - q00[c], q00[c]);
      const float bot = fmaf(fx, q11[c] - q10[c], q10[c]);
      v[c] = fmaf(fy, bot - top, top);
    }
    t = v[0];
    sx = v[1];
    sy = v[2];
  }
  t = fminf(fmaxf(t, 0.f), 1.f);
  const double a = 1.0 / m.max_depth, b = 1.0 / m.min_depth;
  const float depth = (float)(1.0 / (a + (b - a) * (double)t));
  sx = fminf(fmaxf(sx, -4.f), 4.f);
  sy = fminf(fmaxf(sy, -4.f), 4.f);
  const float3 v = plane_from_depth_normal((float)j, (float)i, m.Kinv_d, depth,
                                           make_float3(sx, sy, -1.f));
  float* planes = m.prop_init;
  planes[3 * (size_t)k] = v.x;
  planes[3 * (size_t)k + 1] = v.y;
  planes[3 * (size_t)k + 2] = v.z;
}

// PatchMatch result -> training target (t, sx, sy, weight) on the proposal
// grid of stride S: grid point (ys, xs) takes pixel (S ys, S xs).
__global__ void planes_to_target_kernel(const float4* __restrict__ state,
                                        const float* __restrict__ score, int W, int H, int S,
                                        const MapDev* __restrict__ maps, int map,
                                        float min_score, float* __restrict__ target) {
  const MapDev& m = maps[map];
  const int Ws = (W + S - 1) / S, Hs = (H + S - 1) / S;
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= Ws * Hs) return;
  const int ys = g / Ws, xs = g - ys * Ws;
  const size_t k = (size_t)(S * ys) * W + S * xs;
  const float4 s = state[k];
  float4 tg = make_float4(0.f, 0.f, 0.f, 0.f);
  if (s.w > 0.f && s.z != 0.f && score[k] >= min_score) {
    const double a = 1.0 / m.max_depth, b = 1.0 / m.min_depth;
    const float t = (float)((1.0 / s.w - a) / (b - a));
    tg = make_float4(fminf(fmaxf(t, 0.f), 1.f), fminf(fmaxf(-s.x / s.z, -4.f), 4.f),
                     fminf(fmaxf(-s.y / s.z, -4.f), 4.f), 1.f);
  }
  *reinterpret_cast<float4*>(target + 4 * (size_t)g) = tg;
}

// ------------------------------------------------------------ launchers
template <int CIN, int COUT>
static cudaError_t conv_fwd_t(const ConvArgs& c, cudaStream_t s) {
  const long long blocks = (c.n_pix + 63) / 64;
  conv3x3_fwd_kernel<CIN, COUT><<<(unsigned)blocks, 128, 0, s>>>(c.x, c.w, c.bias, c.n_pix, c.H, c.W,
                                                                 c.relu, c.y, c.y32);
  return cudaGetLastError();
}
template <int CIN, int COUT>
static cudaError_t conv_bwd_t(const ConvArgs& c, __nv_bfloat16* wt_scratch, cudaStream_t s) {
  constexpr int COUTP = ((COUT + 15) / 16) * 16;
  const long long blocks = (c.n_pix + 63) / 64;
  if (c.dx) {
    const int nt = CIN * 9 * COUTP;
    transpose_weights_kernel<<<(nt + 255) / 256, 256, 0, s>>>(c.w, CIN, COUT, COUTP, wt_scratch);
    conv3x3_bwd_data_kernel<CIN, COUT><<<(unsigned)blocks, 128, 0, s>>>(c.dy, wt_scratch, c.x_mask,
                                                                        c.n_pix, c.H, c.W, c.dx);
  }
  const int ppb = 1024;
  const long long wblocks = (c.n_pix + ppb - 1) / ppb;
  conv3x3_bwd_weight_kernel<CIN, COUT><<<(unsigned)wblocks, 128, 0, s>>>(c.dy, c.x, c.n_pix, c.H, c.W,
                                                                         ppb, c.dw, c.db);
  return cudaGetLastError();
}

template <int NP>
static cudaError_t conv_fwd_tc(const ConvArgs& c, cudaStream_t s) {
  auto kern = conv3x3_fwd_tc_kernel<NP>;
  const size_t smem = tc::smem_bytes(NP);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  // Prefer the largest shared-memory carveout so that several CTAs fit per
  // SM from the first launch on (the grid is sized from the occupancy).
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                           cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, smem);
  if (e != cudaSuccess) return e;
  const long long n_img = c.n_pix / ((long long)c.H * c.W);
  const long long tiles = n_img * ((c.H + tc::kTR - 1) / tc::kTR) * ((c.W + tc::kTC - 1) / tc::kTC);
  // The occupancy query has returned one CTA per SM on some calls, where 4
  // fit (registers) and 5 (shared memory).  The CTAs do not wait on one
  // another, so the grid follows the launch bound (4 per SM) at least: any
  // that do not fit run when a slot frees.
  const long long grid = std::min<long long>(tiles, (long long)std::max(per_sm, 4) * sms);
  kern<<<(unsigned)grid, 128, smem, s>>>(c.x, c.w, c.bias, c.H, c.W, c.cout, c.relu, c.y, c.y32,
                                         tiles, c.x_mask);
  return cudaGetLastError();
}

cudaError_t conv3x3_forward(const ConvArgs& c, cudaStream_t s) {
  if (c.cin == 32 && c.cout == 32) return conv_fwd_tc<32>(c, s);
  if (c.cin == 32 && c.cout == 4) return conv_fwd_tc<16>(c, s);
  return cudaErrorInvalidValue;
}

cudaError_t conv3x3_forward_mma_sync(const ConvArgs& c, cudaStream_t s) {
  if (c.cin == 32 && c.cout == 32) return conv_fwd_t<32, 32>(c, s);
  if (c.cin == 32 && c.cout == 4) return conv_fwd_t<32, 4>(c, s);
  return cudaErrorInvalidValue;
}

int take_tc_error() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, tc::g_error, sizeof(int)) != cudaSuccess) return -1;
  if (v) {
    const int zero = 0;
    cudaMemcpyToSymbol(tc::g_error, &zero, sizeof(int));
  }
  return v;
}
cudaError_t conv3x3_backward(const ConvArgs& c, __nv_bfloat16* wt_scratch, cudaStream_t s) {
  if (c.cin == 32 && c.cout == 32) return conv_bwd_t<32, 32>(c, wt_scratch, s);
  if (c.cin == 32 && c.cout == 4) return conv_bwd_t<32, 4>(c, wt_scratch, s);
  return cudaErrorInvalidValue;
}

template <int N>
static cudaError_t conv_bwd_weight_tc(const ConvArgs& c, cudaStream_t s) {
  auto kern = conv3x3_bwd_weight_tc_kernel<N>;
  const size_t smem = tcw::smem_bytes(N);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long n_img = c.n_pix / ((long long)c.H * c.W);
  const long long tiles = n_img * ((c.H + tc::kTR - 1) / tc::kTR) * ((c.W + tc::kTC - 1) / tc::kTC);
  // Two CTAs per SM: each adds its sums to dw once, so fewer CTAs also
  // means fewer atomics.
  const long long grid = std::min<long long>(tiles, 2LL * sms);
  if (grid <= 0) return cudaSuccess;
  kern<<<(unsigned)grid, 128, smem, s>>>(c.dy, c.cout, c.cout, c.x, c.H, c.W, tiles, c.dw, c.db);
  return cudaGetLastError();
}

cudaError_t conv3x3_backward_tc(const ConvArgs& c, __nv_bfloat16* wt_scratch,
                                __nv_bfloat16* dy_pad, cudaStream_t s) {
  if (c.cin != 32 || (c.cout != 32 && c.cout != 4)) return cudaErrorInvalidValue;
  cudaError_t e = c.cout == 32 ? conv_bwd_weight_tc<32>(c, s) : conv_bwd_weight_tc<16>(c, s);
  if (e != cudaSuccess || !c.dx) return e;
  // Backward-data: the forward kernel on the gradient (32 channels) with the
  // flipped weights, no bias, the ReLU mask of the layer's input.
  flip_weights_kernel<<<(32 * 288 + 255) / 256, 256, 0, s>>>(c.w, c.cout, wt_scratch);
  const __nv_bfloat16* g32 = c.dy;
  if (c.cout != 32) {
    pad_channels_kernel<<<(unsigned)((c.n_pix * 32 + 255) / 256), 256, 0, s>>>(c.dy, c.cout,
                                                                               c.n_pix, dy_pad);
    g32 = dy_pad;
  }
  ConvArgs f{};
  f.x = g32;
  f.w = wt_scratch;
  f.bias = nullptr;
  f.n_pix = c.n_pix;
  f.H = c.H;
  f.W = c.W;
  f.cin = 32;
  f.cout = 32;
  f.relu = 0;
  f.y = c.dx;
  f.x_mask = c.x_mask;
  return conv_fwd_tc<32>(f, s);
}
template <int L, int S>
static cudaError_t sweep_l(const LaunchArgs& a, __nv_bfloat16* feat, long long map_stride,
                           int n_planes, cudaStream_t s) {
  // a.tiles: (bx / L) x by grid points per block on the stride-S grid.
  const size_t smem = sizeof(float) * (S * (a.bx / L) + 6) * (S * a.by + 6);
  sweep_features_kernel<L, S><<<a.n_tiles, dim3(a.bx, a.by), smem, s>>>(
      a.maps, a.views, a.pairs, a.tiles, feat, map_stride, n_planes);
  return cudaGetLastError();
}
template <int S>
static cudaError_t sweep_s(const LaunchArgs& a, __nv_bfloat16* feat, long long map_stride,
                           int n_planes, cudaStream_t s) {
  switch (a.p.variant) {
    case 1: return sweep_l<1, S>(a, feat, map_stride, n_planes, s);
    case 2: return sweep_l<2, S>(a, feat, map_stride, n_planes, s);
    case 4: return sweep_l<4, S>(a, feat, map_stride, n_planes, s);
    case 8: return sweep_l<8, S>(a, feat, map_stride, n_planes, s);
  }
  return cudaErrorInvalidValue;
}
cudaError_t launch_sweep(const LaunchArgs& a, __nv_bfloat16* feat, long long map_stride,
                         int n_planes, int stride, cudaStream_t s) {
  if (a.n_tiles == 0) return cudaSuccess;
  if (stride == 1) return sweep_s<1>(a, feat, map_stride, n_planes, s);
  if (stride == 2) return sweep_s<2>(a, feat, map_stride, n_planes, s);
  if (stride == 4) return sweep_s<4>(a, feat, map_stride, n_planes, s);
  if (stride == 8) return sweep_s<8>(a, feat, map_stride, n_planes, s);
  return cudaErrorInvalidValue;
}
cudaError_t launch_l1_loss(const float* pred, const float* target, long long n_pix,
                           float normal_weight, __nv_bfloat16* dpred, float* loss_sum, float* count,
                           cudaStream_t s) {
  l1_loss_kernel<<<(unsigned)((n_pix + 255) / 256), 256, 0, s>>>(pred, target, n_pix, normal_weight,
                                                                 dpred, loss_sum, count);
  return cudaGetLastError();
}
cudaError_t launch_adam(float* w, float* m, float* v, const float* grad, int n, const float* count,
                        float lr, float b1, float b2, float eps, float bc1, float bc2,
                        __nv_bfloat16* w16, cudaStream_t s) {
  adam_kernel<<<(n + 255) / 256, 256, 0, s>>>(w, m, v, grad, n, count, lr, b1, b2, eps, bc1, bc2, w16);
  return cudaGetLastError();
}
cudaError_t launch_output_to_planes(const float* out, int W, int H, const MapDev* maps, int map,
                                    float* planes, cudaStream_t s) {
  output_to_planes_kernel<<<(W * H + 255) / 256, 256, 0, s>>>(out, W, H, maps, map, planes);
  return cudaGetLastError();
}
cudaError_t launch_planes_to_target(const float4* state, const float* score, int W, int H,
                                    int stride, const MapDev* maps, int map, float min_score,
                                    float* target, cudaStream_t s) {
  const int n = ((W + stride - 1) / stride) * ((H + stride - 1) / stride);
  planes_to_target_kernel<<<(n + 255) / 256, 256, 0, s>>>(state, score, W, H, stride, maps, map,
                                                          min_score, target);
  return cudaGetLastError();
}
cudaError_t launch_proposal_to_planes(const float* out, const MapDev* maps, int n_maps,
                                      int max_pixels, cudaStream_t s) {
  if (n_maps == 0) return cudaSuccess;
  const dim3 grid((unsigned)((max_pixels + 255) / 256), (unsigned)n_maps);
  proposal_to_planes_kernel<<<grid, 256, 0, s>>>(out, maps);
  return cudaGetLastError();
}

}  // namespace dn
