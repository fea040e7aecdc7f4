// Learned proposal network: a small BF16 encoder-decoder that predicts an initial plane (inverse depth, normal) and a
// confidence per pixel from the reference image and a plane-sweep NCC cost volume.  No reference counterpart: it is
// the "learned proposal" addition to the PatchStereo engine.  Training and inference run on hand-written kernels:
//   * 3×3 convolution forward as an implicit GEMM on the tensor cores (mma.sync m16n8k16, BF16 operands, FP32
//     accumulation), bias and ReLU fused into the epilogue; the data gradient is the same kernel run with the
//     weights flipped in space and transposed in channels;
//   * 3×3 convolution weight gradient as a split-K implicit GEMM (tensor cores, FP32 atomics across pixel chunks);
//   * 2×2 average pooling, nearest 2× upsampling, channel concat and their gradients, the loss and its gradient,
//     AdamW on FP32 master weights with BF16 copies for the forward pass.
// Layout: activations NHWC in BF16 with channel counts that are multiples of 16; weights [Cout][9][Cin] (K-major).
//
// Network (channels per level 32/64/96/128):
//   e0: 48->32->32 | pool | e1: 32->64->64 | pool | e2: 64->96->96 | pool | e3: 96->128->128
//   d2: up(e3) ++ e2 (224) -> 96 | d1: up(d2) ++ e1 (160) -> 64 | d0: up(d1) ++ e0 (96) -> 32 | head: 32 -> 8 (5 used)
// Outputs: o0 = logit of the normalised inverse depth, o1..o3 = normal direction, o4 = logit of the confidence.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <new>
#include <string>
#include <vector>

#include "../../include/patchstereo.h"
#include "ps_cnn.h"
#include "ps_types.h"

typedef __nv_bfloat16 bf16;

namespace ps_cnn {

// ------------------------------------------------------------------------------------------- tensor-core tiles
// Convolution as an implicit GEMM: C[p][co] = sum_{tap, ci} X[p shifted by tap][ci] * W[co][tap][ci] (M = pixels,
// N = cout, K = 9·cin) on mma.sync m16n8k16 (bf16 operands, f32 accumulators).  Weight-gradient tile (k_conv_wgrad):
// 128 threads, 64 × 64 outputs, K in chunks of 16 pixels; warps 2 × 2, each 32 × 32 = 2 (m16) × 4 (n8) fragments.
constexpr int CM = 64, CN = 64, CK = 16, CPAD = 8;

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

struct ConvArgs {
  const bf16* x;   // [B][H][W][cin_stride], channels [cin_off, cin_off+cin) are read
  const bf16* w;   // [cout][9][cin]
  const float* bias;  // [cout] or null
  bf16* y;         // [B][H][W][cout] (bf16 output) or null
  float* yf;       // [B][H][W][cout] (f32 output) or null
  int B, H, W, cin, cin_stride, cin_off, cout;
  int relu;
  // Virtual "upsample + concatenate" input (k_conv2 only; x2 == null: off): input channels [0, split) are x at half
  // resolution [B][H/2][W/2][cin_stride] read at (y/2, x/2) (nearest 2× upsampling), channels [split, cin) are
  // x2 [B][H][W][x2_stride] (the skip connection).  split is a multiple of 8.
  const bf16* x2;
  int split, x2_stride;
};


// ------------------------------------------------------------------------------------------- conv forward, halo-tiled
// The production convolution.  A CTA (8 warps) computes an 8 × 16 pixel output tile for BN output channels.  For each
// chunk of 32 input channels it stages, with cp.async into a double buffer, the (8+2) × (16+2) halo of the input tile
// and the chunk's weights for all 9 taps; every tap then reads its shifted A operand from the same halo copy.  Warp w
// owns output row w of the tile (16 pixels = one m16 fragment) × BN columns; fragments come from shared memory through
// ldmatrix (rows padded to 80 bytes, so the 8 row addresses of a matrix hit distinct banks).  Out-of-image halo pixels
// and input channels beyond cin are zero-filled by the copy itself (source size 0).
constexpr int HT_H = 8, HT_W = 16, HALO_W = HT_W + 2, HALO_PX = (HT_H + 2) * HALO_W;
constexpr int KC = 32, KCP = 40;  // channels per stage, padded row length (bf16)

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void ldsm_x4(uint32_t* r, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x2(uint32_t* r, const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r[0]), "=r"(r[1]) : "r"(smem_u32(p)));
}

template <int BN>
constexpr size_t conv2_smem() {
  return (size_t)2 * (HALO_PX * KCP + 9 * BN * KCP) * sizeof(bf16);
}

template <int BN>
__global__ void __launch_bounds__(256) k_conv2(ConvArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  bf16* halo = reinterpret_cast<bf16*>(smraw);  // [2][HALO_PX][KCP]
  bf16* wsm = halo + 2 * HALO_PX * KCP;         // [2][9][BN][KCP]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tiles_x = (a.W + HT_W - 1) / HT_W, tiles_y = (a.H + HT_H - 1) / HT_H;
  int t = blockIdx.x;
  const int b = t / (tiles_x * tiles_y);
  t -= b * tiles_x * tiles_y;
  const int ty0 = (t / tiles_x) * HT_H, tx0 = (t % tiles_x) * HT_W;
  const int n0 = blockIdx.y * BN;
  const int nchunks = (a.cin + KC - 1) / KC;

  auto load_stage = [&](int stage, int kc) {
    const int c0 = kc * KC;
    for (int i = tid; i < HALO_PX * 4; i += 256) {
      const int px = i >> 2, seg = i & 3;
      const int hy = px / HALO_W, hx = px - hy * HALO_W;
      const int gy = ty0 + hy - 1, gx = tx0 + hx - 1, ch = c0 + seg * 8;
      const bool ok = gy >= 0 && gy < a.H && gx >= 0 && gx < a.W && ch < a.cin;
      const bf16* src = a.x;
      if (ok) {
        if (!a.x2)
          src = a.x + (((long long)b * a.H + gy) * a.W + gx) * a.cin_stride + a.cin_off + ch;
        else if (ch < a.split)
          src = a.x + (((long long)b * (a.H >> 1) + (gy >> 1)) * (a.W >> 1) + (gx >> 1)) * a.cin_stride + ch;
        else
          src = a.x2 + (((long long)b * a.H + gy) * a.W + gx) * a.x2_stride + (ch - a.split);
      }
      cp_async16(halo + ((size_t)stage * HALO_PX + px) * KCP + seg * 8, src, ok ? 16 : 0);
    }
    for (int i = tid; i < 9 * BN * 4; i += 256) {
      const int seg = i & 3, r = i >> 2;
      const int n = r % BN, tap = r / BN;
      const int co = n0 + n, ch = c0 + seg * 8;
      const bool ok = co < a.cout && ch < a.cin;
      const bf16* src = ok ? a.w + ((long long)co * 9 + tap) * a.cin + ch : a.w;
      cp_async16(wsm + (((size_t)stage * 9 + tap) * BN + n) * KCP + seg * 8, src, ok ? 16 : 0);
    }
    cp_async_commit();
  };

  float acc[BN / 8][4];
#pragma unroll
  for (int j = 0; j < BN / 8; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[j][e] = 0.f;

  load_stage(0, 0);
  for (int kc = 0; kc < nchunks; ++kc) {
    if (kc + 1 < nchunks) {
      load_stage((kc + 1) & 1, kc + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int st = kc & 1;
    const bf16* hs = halo + (size_t)st * HALO_PX * KCP;
    const bf16* ws = wsm + (size_t)st * 9 * BN * KCP;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int dy = tap / 3, dx = tap - dy * 3;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) {
        uint32_t af[4];
        ldsm_x4(af, hs + ((warp + dy) * HALO_W + (lane & 15) + dx) * KCP + ks * 16 + (lane >> 4) * 8);
        const bf16* wt = ws + (size_t)tap * BN * KCP + ks * 16 + ((lane >> 3) & 1) * 8;
#pragma unroll
        for (int j = 0; j < BN / 8; j += 2) {
          if (j + 1 < BN / 8) {
            uint32_t bq[4];
            ldsm_x4(bq, wt + (j * 8 + (lane >> 4) * 8 + (lane & 7)) * KCP);
            mma_bf16(acc[j], af, bq);
            mma_bf16(acc[j + 1], af, bq + 2);
          } else {
            uint32_t bq[2];
            ldsm_x2(bq, wt + (j * 8 + (lane & 7)) * KCP);
            mma_bf16(acc[j], af, bq);
          }
        }
      }
    }
    __syncthreads();  // every warp is done with this stage before the next prefetch overwrites it
  }
  // epilogue: rows g and g+8 of the m16 fragment are output columns tx0+g and tx0+g+8 of tile row `warp`
  const int g = lane >> 2, tq = lane & 3, oy = ty0 + warp;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int ox = tx0 + g + h * 8;
    if (oy >= a.H || ox >= a.W) continue;
    const long long p = ((long long)b * a.H + oy) * a.W + ox;
#pragma unroll
    for (int j = 0; j < BN / 8; ++j) {
      const int co = n0 + j * 8 + tq * 2;  // cout is a multiple of 8: co + 1 < cout whenever co < cout
      if (co >= a.cout) continue;
      float v0 = acc[j][h * 2] + (a.bias ? a.bias[co] : 0.f);
      float v1 = acc[j][h * 2 + 1] + (a.bias ? a.bias[co + 1] : 0.f);
      if (a.relu) {
        v0 = fmaxf(v0, 0.f);
        v1 = fmaxf(v1, 0.f);
      }
      if (a.y) *reinterpret_cast<__nv_bfloat162*>(a.y + p * a.cout + co) = __floats2bfloat162_rn(v0, v1);
      if (a.yf) *reinterpret_cast<float2*>(a.yf + p * a.cout + co) = make_float2(v0, v1);
    }
  }
}

// ------------------------------------------------------------------------------------------- conv forward on tcgen05
// Inference and training convolutions with cout = N in {32, 64, 96, 128} on the 5th-generation tensor cores.  A CTA
// (4 warps) computes R = 4 output rows × 128 pixels × N channels; the R accumulators D_r[128 × N] (f32) sit side by side
// in tensor memory (columns r·N .. r·N + N).  Per chunk of KCH input channels the CTA stages, with cp.async into a
// double buffer,
//   * the R + 2 input rows y0-1 .. y0+R over pixels x0-1 .. x0+128 in the canonical K-major layout without swizzle,
//     [row][kgroup (8 channels)][pixel][8 channels] = 16 bytes per (pixel, kgroup): the A operand of output row r and
//     tap (dy, dx) is input row r + dy with its start address moved by dx pixels (16 bytes), so nothing is re-laid;
//   * the chunk's weights of the 9 taps as [tap][kgroup][n][8 channels] (the B operand, shared by the R rows).
// One thread issues R × 9 taps × KCH/16 tcgen05.mma (M = 128, N, K = 16, bf16 -> f32) and commits them to the stage's
// mbarrier; refilling that stage waits on it.  The epilogue reads each D_r with tcgen05.ld (warp w owns TMEM lanes
// 32w .. 32w+31 = pixels), adds the bias, applies ReLU and stores bf16 or f32.  Every wait is bounded: on expiry the
// kernel counts it in g_conv5_timeouts and skips the remaining work (the host reports invalid results); every CTA frees
// its tensor memory before it exits.
constexpr int T5_PX = 128, T5_ROWPX = T5_PX + 2;  // pixels per row segment, staged pixels per row
constexpr unsigned long long T5_WAIT_NS = 200000000ull;     // bound on one mbarrier wait (a chunk takes microseconds)
constexpr long long T5_SPIN = 1ll << 24;                     // and on its polls
__device__ unsigned int g_conv5_timeouts = 0;
__device__ int g_conv5_stall = 0;  // failure test: the issuing thread commits nothing, so the bounded waits run out

template <int N>
struct Conv5Cfg {
  static constexpr int R = N <= 32 ? 2 : 4;      // output rows per CTA (two CTAs per SM for N = 32)
  static constexpr int KCH = N <= 64 ? 32 : 16;  // input channels per stage
  static constexpr int KG = KCH / 8;             // kgroups per stage
  static constexpr size_t in_bytes = (size_t)(R + 2) * KG * T5_ROWPX * 16;
  static constexpr size_t w_bytes = (size_t)9 * KG * N * 16;
  static constexpr size_t smem = 2 * (in_bytes + w_bytes) + 64;
  static constexpr int cols = R * N <= 64 ? 64 : (R * N <= 128 ? 128 : (R * N <= 256 ? 256 : 512));  // 2^k >= R·N
};

// Shared-memory matrix descriptor, K-major, no swizzle (16-byte rows in groups of 8 at `sbo`, K chunks at `lbo`).
__device__ __forceinline__ uint64_t umma_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100; base offset 0, layout type 0 (no swizzle)
  return d;
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count));
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Waits for the completion of the phase with the given parity; false once 200 ms (or 2^24 polls) have passed.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  const unsigned long long t0 = global_ns();
  for (long long i = 0; i < T5_SPIN; ++i) {
    if ((i & 255) == 255 && global_ns() - t0 > T5_WAIT_NS) return false;
    unsigned done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

template <int N>
__global__ void __launch_bounds__(128, 1) k_conv5(ConvArgs a) {
  using Cfg = Conv5Cfg<N>;
  constexpr int KCH = Cfg::KCH, KG = Cfg::KG, T5_R = Cfg::R;
  extern __shared__ __align__(128) unsigned char sm5[];
  unsigned char* in_s = sm5;                        // [2][R+2][KG][130][16 B]
  unsigned char* w_s = sm5 + 2 * Cfg::in_bytes;     // [2][9][KG][N][16 B]
  unsigned char* misc = w_s + 2 * Cfg::w_bytes;     // mbarriers, TMEM address, flags
  const unsigned bar0 = smem_u32(misc), bar1 = smem_u32(misc + 8);
  volatile unsigned* tmem_slot = reinterpret_cast<volatile unsigned*>(misc + 16);
  volatile int* fail_flag = reinterpret_cast<volatile int*>(misc + 20);
  volatile int* last_commit = reinterpret_cast<volatile int*>(misc + 24);  // last chunk whose MMAs were committed
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int segs = (a.W + T5_PX - 1) / T5_PX, bands = (a.H + T5_R - 1) / T5_R;
  int t = blockIdx.x;
  const int seg = t % segs;
  t /= segs;
  const int y0 = (t % bands) * T5_R, b = t / bands;
  const int x0 = seg * T5_PX;
  const int nchunks = (a.cin + KCH - 1) / KCH;

  if (warp == 0) {  // tensor memory for the accumulators (warp-wide)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(misc + 16)),
                 "r"(Cfg::cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  if (tid == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    *fail_flag = *(volatile unsigned*)&g_conv5_timeouts != 0;  // after any expired wait, skip all work quickly
    *last_commit = -1;
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const unsigned tmem = *tmem_slot;

  auto load_stage = [&](int stage, int kc) {
    const int c0 = kc * KCH;
    unsigned char* is = in_s + (size_t)stage * Cfg::in_bytes;
    for (int i = tid; i < (T5_R + 2) * KG * T5_ROWPX; i += 128) {
      const int px = i % T5_ROWPX, g = (i / T5_ROWPX) % KG, r = i / (T5_ROWPX * KG);
      const int gy = y0 + r - 1, gx = x0 + px - 1, ch = c0 + g * 8;
      const bool ok = gy >= 0 && gy < a.H && gx >= 0 && gx < a.W && ch < a.cin;
      const bf16* src = a.x;
      if (ok) {
        if (!a.x2)
          src = a.x + (((long long)b * a.H + gy) * a.W + gx) * a.cin_stride + a.cin_off + ch;
        else if (ch < a.split)
          src = a.x + (((long long)b * (a.H >> 1) + (gy >> 1)) * (a.W >> 1) + (gx >> 1)) * a.cin_stride + ch;
        else
          src = a.x2 + (((long long)b * a.H + gy) * a.W + gx) * a.x2_stride + (ch - a.split);
      }
      cp_async16(is + ((size_t)(r * KG + g) * T5_ROWPX + px) * 16, src, ok ? 16 : 0);
    }
    unsigned char* ws = w_s + (size_t)stage * Cfg::w_bytes;
    for (int i = tid; i < 9 * KG * N; i += 128) {
      const int n = i % N, g = (i / N) % KG, tap = i / (N * KG);
      const int ch = c0 + g * 8;
      const bool ok = n < a.cout && ch < a.cin;
      const bf16* src = ok ? a.w + ((long long)n * 9 + tap) * a.cin + ch : a.w;
      cp_async16(ws + ((size_t)(tap * KG + g) * N + n) * 16, src, ok ? 16 : 0);
    }
    cp_async_commit();
  };

  // instruction descriptor: f32 accumulator, bf16 A and B, both K-major, N, M = 128
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  load_stage(0, 0);
  for (int kc = 0; kc < nchunks; ++kc) {
    const int st = kc & 1;
    if (kc + 1 < nchunks) {
      // the stage about to be refilled held chunk kc-1: its MMAs must have finished reading it
      if (kc >= 1 && !*fail_flag && !mbar_wait(st ? bar0 : bar1, ((kc - 1) >> 1) & 1)) {
        *fail_flag = 1;
        atomicAdd(&g_conv5_timeouts, 1u);
      }
      load_stage((kc + 1) & 1, kc + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // cp.async data -> tensor-core operand reads
    __syncthreads();
    if (tid == 0 && !*fail_flag && !*(volatile int*)&g_conv5_stall) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
      const unsigned ib = smem_u32(in_s + (size_t)st * Cfg::in_bytes);
      const unsigned wb = smem_u32(w_s + (size_t)st * Cfg::w_bytes);
#pragma unroll 1
      for (int tap = 0; tap < 9; ++tap) {
        const int dy = tap / 3, dx = tap - dy * 3;
#pragma unroll
        for (int ks = 0; ks < KCH / 16; ++ks) {
          const unsigned baddr = wb + (unsigned)(((tap * KG + 2 * ks) * N) * 16);
          const uint64_t bd = umma_desc(baddr, N * 16, 128);
          const unsigned acc = (kc | tap | ks) != 0;
#pragma unroll
          for (int r = 0; r < T5_R; ++r) {
            const unsigned aaddr = ib + (unsigned)((((r + dy) * KG + 2 * ks) * T5_ROWPX + dx) * 16);
            const uint64_t ad = umma_desc(aaddr, T5_ROWPX * 16, 128);
            asm volatile(
                "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(
                    tmem + (unsigned)(r * N)),
                "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                       st ? bar1 : bar0)
                   : "memory");
      *last_commit = kc;
    }
  }
  // the last commit covers every MMA this CTA issued: wait for it before reading or freeing tensor memory
  __syncthreads();
  const int lc = *last_commit;
  const bool failed = *fail_flag;
  const bool done = !failed && lc >= 0 && mbar_wait((lc & 1) ? bar1 : bar0, (lc >> 1) & 1);
  // one decision for the whole CTA: the tensor-memory loads below are warp-collective
  const bool ok = __syncthreads_and(done ? 1 : 0) && lc == nchunks - 1;
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const int px = x0 + warp * 32 + lane;
  if (ok) {
#pragma unroll 1
    for (int r = 0; r < T5_R; ++r) {
      const int y = y0 + r;
#pragma unroll 1
      for (int c0 = 0; c0 < N; c0 += 32) {
        uint32_t v32[32];
        const unsigned taddr = tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(r * N + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,"
            "%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
            : "=r"(v32[0]), "=r"(v32[1]), "=r"(v32[2]), "=r"(v32[3]), "=r"(v32[4]), "=r"(v32[5]), "=r"(v32[6]),
              "=r"(v32[7]), "=r"(v32[8]), "=r"(v32[9]), "=r"(v32[10]), "=r"(v32[11]), "=r"(v32[12]), "=r"(v32[13]),
              "=r"(v32[14]), "=r"(v32[15]), "=r"(v32[16]), "=r"(v32[17]), "=r"(v32[18]), "=r"(v32[19]),
              "=r"(v32[20]), "=r"(v32[21]), "=r"(v32[22]), "=r"(v32[23]), "=r"(v32[24]), "=r"(v32[25]),
              "=r"(v32[26]), "=r"(v32[27]), "=r"(v32[28]), "=r"(v32[29]), "=r"(v32[30]), "=r"(v32[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (px < a.W && y < a.H) {
          const long long p = ((long long)b * a.H + y) * a.W + px;
#pragma unroll
          for (int j = 0; j < 32; j += 8) {
            float v[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
              v[e] = __uint_as_float(v32[j + e]) + (a.bias ? a.bias[c0 + j + e] : 0.f);
              if (a.relu) v[e] = fmaxf(v[e], 0.f);
            }
            if (a.y) {
              uint4 o;
              __nv_bfloat162* h2 = reinterpret_cast<__nv_bfloat162*>(&o);
#pragma unroll
              for (int e = 0; e < 4; ++e) h2[e] = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
              *reinterpret_cast<uint4*>(a.y + p * a.cout + c0 + j) = o;
            }
            if (a.yf) {
              float4* f = reinterpret_cast<float4*>(a.yf + p * a.cout + c0 + j);
              f[0] = make_float4(v[0], v[1], v[2], v[3]);
              f[1] = make_float4(v[4], v[5], v[6], v[7]);
            }
          }
        }
      }
    }
  }
  if (tid == 0 && !ok && !failed) atomicAdd(&g_conv5_timeouts, 1u);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(Cfg::cols));
}

// ------------------------------------------------------------------------------------------- conv weight gradient
// dW[co][tap][ci] += sum_p dY[p][co] * X[p shifted by tap][ci];  M = Cout, N = 9·Cin (n = tap·Cin + ci), K = pixels.
// Each CTA reduces a chunk of `pix_per_cta` pixels and adds its 64×64 tile into dW with FP32 atomics.
struct WgradArgs {
  const bf16* dy;  // [P][cout]
  const bf16* x;   // [B][H][W][cin_stride] (+cin_off)
  float* dw;       // [cout][9][cin]
  int B, H, W, cin, cin_stride, cin_off, cout, pix_per_cta;
};

__global__ void __launch_bounds__(128) k_conv_wgrad(WgradArgs a) {
  __shared__ __align__(16) bf16 As[CM][CK + CPAD];  // [co][p]
  __shared__ __align__(16) bf16 Bs[CN][CK + CPAD];  // [n][p]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int co0 = blockIdx.x * CM;
  const int nk = 9 * a.cin;
  const int n0 = blockIdx.y * CN;
  const long long P = (long long)a.B * a.H * a.W;
  const long long pbeg = (long long)blockIdx.z * a.pix_per_cta;
  const long long pend = min(P, pbeg + a.pix_per_cta);
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.f;
  for (long long pc = pbeg; pc < pend; pc += CK) {
    // A: As[co][pp] = dY[pc+pp][co0+co]; 64 × 16 -> each thread 8 values
    for (int e = tid; e < CM * CK; e += 128) {
      const int pp = e / CM, co = e % CM;
      const long long p = pc + pp;
      bf16 v = __float2bfloat16(0.f);
      if (p < pend && co0 + co < a.cout) v = a.dy[p * a.cout + co0 + co];
      As[co][pp] = v;
    }
    // B: Bs[n][pp] = X[pc+pp shifted by tap(n)][ci(n)]
    for (int e = tid; e < CN * CK; e += 128) {
      const int pp = e / CN, nn = e % CN;
      const long long p = pc + pp;
      const int n = n0 + nn;
      bf16 v = __float2bfloat16(0.f);
      if (p < pend && n < nk) {
        const int tap = n / a.cin, ci = n - tap * a.cin;
        const int b = (int)(p / ((long long)a.H * a.W));
        const int rem = (int)(p - (long long)b * a.H * a.W);
        const int y = rem / a.W + tap / 3 - 1, x = rem % a.W + tap % 3 - 1;
        if (y >= 0 && y < a.H && x >= 0 && x < a.W)
          v = a.x[(((long long)b * a.H + y) * a.W + x) * a.cin_stride + a.cin_off + ci];
      }
      Bs[nn][pp] = v;
    }
    __syncthreads();
    const int g = lane >> 2, t = lane & 3;
    uint32_t af[2][4], bfr[4][2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int r = wm * 32 + i * 16 + g;
      af[i][0] = *(const uint32_t*)&As[r][t * 2];
      af[i][1] = *(const uint32_t*)&As[r + 8][t * 2];
      af[i][2] = *(const uint32_t*)&As[r][t * 2 + 8];
      af[i][3] = *(const uint32_t*)&As[r + 8][t * 2 + 8];
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = wn * 32 + j * 8 + g;
      bfr[j][0] = *(const uint32_t*)&Bs[c][t * 2];
      bfr[j][1] = *(const uint32_t*)&Bs[c][t * 2 + 8];
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
    __syncthreads();
  }
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int co = co0 + wm * 32 + i * 16 + g + h * 8;
      if (co >= a.cout) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int n = n0 + wn * 32 + j * 8 + t * 2 + e;
          if (n < nk) atomicAdd(a.dw + (long long)co * nk + n, acc[i][j][h * 2 + e]);
        }
    }
}

// ------------------------------------------------------------------------------------------- small kernels
// W' [cin][9][cout] = W [cout][8 - tap][cin] (bf16): the data gradient of a 3×3 "same" convolution is the
// convolution of dY with the spatially flipped, channel-transposed weights.
__global__ void k_flip_weights(const bf16* w, bf16* wt, int cout, int cin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cout * 9 * cin) return;
  const int ci = i % cin, tap = (i / cin) % 9, co = i / (9 * cin);
  wt[((long long)ci * 9 + (8 - tap)) * cout + co] = w[i];
}

// dY ⊙ (Y > 0) for a ReLU layer (in place on dY).
__global__ void k_relu_bwd(bf16* dy, const bf16* y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!(__bfloat162float(y[i]) > 0.f)) dy[i] = __float2bfloat16(0.f);
}

// db[c] += sum_p dY[p][c]
__global__ void k_bias_grad(const bf16* dy, float* db, long long P, int C) {
  const int c = threadIdx.x % C;
  const int lanes = blockDim.x / C;
  const int sub = threadIdx.x / C;
  if (sub >= lanes) return;
  float s = 0.f;
  for (long long p = (long long)blockIdx.x * lanes + sub; p < P; p += (long long)gridDim.x * lanes)
    s += __bfloat162float(dy[p * C + c]);
  atomicAdd(db + c, s);
}

// 2×2 average pooling (NHWC) and its gradient.
// One thread per 8 channels of an output pixel (16-byte loads and store; C is a multiple of 8).
__global__ void k_pool_fwd(const bf16* x, bf16* y, int B, int H, int W, int C) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int h = H / 2, w = W / 2, C8 = C / 8;
  if (i >= (long long)B * h * w * C8) return;
  const int c = (int)(i % C8) * 8;
  const long long p = i / C8;
  const int xx = p % w, yy = (p / w) % h, b = (int)(p / ((long long)w * h));
  const long long base = (((long long)b * H + 2 * yy) * W + 2 * xx) * C + c;
  const uint4 q[4] = {*(const uint4*)(x + base), *(const uint4*)(x + base + C), *(const uint4*)(x + base + (long long)W * C),
                      *(const uint4*)(x + base + (long long)W * C + C)};
  const bf16* e[4] = {(const bf16*)&q[0], (const bf16*)&q[1], (const bf16*)&q[2], (const bf16*)&q[3]};
  uint4 o;
  bf16* r = (bf16*)&o;
#pragma unroll
  for (int k = 0; k < 8; ++k)
    r[k] = __float2bfloat16(0.25f * (__bfloat162float(e[0][k]) + __bfloat162float(e[1][k]) + __bfloat162float(e[2][k]) +
                                     __bfloat162float(e[3][k])));
  *(uint4*)(y + p * C + c) = o;
}
// dX (full res, C channels) = dY/4 broadcast; `accumulate` adds to dX.
__global__ void k_pool_bwd(const bf16* dy, bf16* dx, int B, int H, int W, int C, int accumulate) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)B * H * W * C) return;
  const int c = i % C;
  const long long p = i / C;
  const int x = p % W, y = (p / W) % H, b = (int)(p / ((long long)W * H));
  float v = 0.25f * __bfloat162float(dy[(((long long)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c]);
  if (accumulate) v += __bfloat162float(dx[i]);
  dx[i] = __float2bfloat16(v);
}
// nearest 2× upsampling of x [B][H/2][W/2][C] into channels [0, C) of y [B][H][W][Cy]; gradient sums the 2×2 block.
__global__ void k_up_fwd(const bf16* x, bf16* y, int B, int H, int W, int C, int Cy) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)B * H * W * C) return;
  const int c = i % C;
  const long long p = i / C;
  const int xx = p % W, yy = (p / W) % H, b = (int)(p / ((long long)W * H));
  y[p * Cy + c] = x[(((long long)b * (H / 2) + yy / 2) * (W / 2) + xx / 2) * C + c];
}
__global__ void k_up_bwd(const bf16* dy, bf16* dx, int B, int H, int W, int C, int Cy) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int h = H / 2, w = W / 2;
  if (i >= (long long)B * h * w * C) return;
  const int c = i % C;
  const long long p = i / C;
  const int xx = p % w, yy = (p / w) % h, b = (int)(p / ((long long)w * h));
  float s = 0.f;
  for (int dy2 = 0; dy2 < 2; ++dy2)
    for (int dx2 = 0; dx2 < 2; ++dx2)
      s += __bfloat162float(dy[(((long long)b * H + 2 * yy + dy2) * W + 2 * xx + dx2) * Cy + c]);
  dx[i] = __float2bfloat16(s);
}
// channel copy: dst[p][doff + c] = src[p][soff + c] (optionally accumulating into dst)
__global__ void k_copy_ch(const bf16* src, int sC, int soff, bf16* dst, int dC, int doff, int C, long long P, int accumulate) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P * C) return;
  const int c = i % C;
  const long long p = i / C;
  float v = __bfloat162float(src[p * sC + soff + c]);
  if (accumulate) v += __bfloat162float(dst[p * dC + doff + c]);
  dst[p * dC + doff + c] = __float2bfloat16(v);
}

__device__ __forceinline__ float sigm(float x) { return 1.f / (1.f + expf(-x)); }

// Loss and gradient of the head output o [P][8] (f32) against labels [P][6]: (target normalised inverse depth
// t* = (1/d* - 1/dmax) / (1/dmin - 1/dmax), normal xyz, valid, target depth d*).  Loss per valid pixel: |t - t*| + (1 - n̂·n*) + 0.5·BCE(conf, |d - d*| < 1 % d*).
// Writes dO (bf16) scaled by 1/valid_count and adds the loss sum and the valid count to stats[0..1].
__global__ void k_loss(const float* o, const float* lab, bf16* dout, float* stats, long long P, float inv_n,
                       float inv_near, float inv_far) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const float* L = lab + p * 6;
  const float* O = o + p * 8;
  float g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  float loss = 0.f, valid = 0.f;
  if (L[4] > 0.5f) {
    valid = 1.f;
    const float t = sigm(O[0]);
    const float dt = t - L[0];
    loss += fabsf(dt);
    g[0] = (dt > 0.f ? 1.f : (dt < 0.f ? -1.f : 0.f)) * t * (1.f - t);
    const float nx = O[1], ny = O[2], nz = O[3];
    const float len = sqrtf(nx * nx + ny * ny + nz * nz) + 1e-6f;
    const float c = (nx * L[1] + ny * L[2] + nz * L[3]) / len;
    loss += 1.f - c;
    // d(-c)/dO_k = -(L_k/len - c·O_k/len²)
    g[1] = -(L[1] / len - c * nx / (len * len));
    g[2] = -(L[2] / len - c * ny / (len * len));
    g[3] = -(L[3] / len - c * nz / (len * len));
    const float inv = inv_far + t * (inv_near - inv_far);
    const float d = 1.f / fmaxf(inv, 1e-9f);
    const float target = fabsf(d - L[5]) < 0.01f * L[5] ? 1.f : 0.f;
    const float cf = sigm(O[4]);
    loss += -0.5f * (target * logf(fmaxf(cf, 1e-7f)) + (1.f - target) * logf(fmaxf(1.f - cf, 1e-7f)));
    g[4] = 0.5f * (cf - target);
  }
  for (int k = 0; k < 8; ++k) dout[p * 8 + k] = __float2bfloat16(g[k] * inv_n);
  if (valid > 0.f) {
    atomicAdd(stats, loss);
    atomicAdd(stats + 1, 1.f);
  }
}

// AdamW on FP32 master weights; refreshes the BF16 copy.
__global__ void k_adamw(float* w, const float* g, float* m, float* v, bf16* wb, long long n, float lr, float b1, float b2,
                        float eps, float wd, float c1, float c2) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float wi = w[i] * (1.f - lr * wd);
  wi -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16(wi);
}

// Head output -> proposal planes (nx, ny, nz, d; all 0 where confidence < thr or the normal is degenerate) and
// confidence for the H × W pixels of a view whose network rows hold Wp pixels.  Normals are flipped toward the camera
// (n · ray < 0 with ray = ((x - cx)/fx, (y - cy)/fy, 1)).
__global__ void k_decode(const float* o, int Wp, int H, int W, float4* planes, float* conf, float inv_near,
                         float inv_far, float thr, float fx, float fy, float cx, float cy, unsigned long long* count) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  bool proposed = false;
  if (x < W && y < H) {
    const float* O = o + ((long long)y * Wp + x) * 8;
    const float t = sigm(O[0]);
    const float inv = inv_far + t * (inv_near - inv_far);
    const float d = 1.f / fmaxf(inv, 1e-9f);
    float nx = O[1], ny = O[2], nz = O[3];
    const float len = sqrtf(nx * nx + ny * ny + nz * nz);
    float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
    const float c = sigm(O[4]);
    if (len > 1e-6f) {
      nx /= len;
      ny /= len;
      nz /= len;
      const float rx = ((float)x - cx) / fx, ry = ((float)y - cy) / fy;
      if (nx * rx + ny * ry + nz > 0.f) {
        nx = -nx;
        ny = -ny;
        nz = -nz;
      }
      if (nx * rx + ny * ry + nz < -1e-3f && c >= thr) out = make_float4(nx, ny, nz, d);
    }
    planes[(long long)y * W + x] = out;
    conf[(long long)y * W + x] = c;
    proposed = out.w > 0.f;
  }
  const unsigned m = __ballot_sync(0xffffffffu, proposed);
  if (count && (threadIdx.x & 31) == 0 && m) atomicAdd(count, (unsigned long long)__popc(m));
}


// Valid-label count (labels [P][6], channel 4 = valid) into *count, for the mean loss.
__global__ void k_count_valid(const float* lab, long long P, float* count) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned m = __ballot_sync(0xffffffffu, p < P && lab[p * 6 + 4] > 0.5f);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(count, (float)__popc(m));
}

// Scales the loss gradient by 1 / count (count read on the device: no host round trip inside a training step).
__global__ void k_scale_grad(bf16* g, long long n, const float* count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float c = *count;
  g[i] = __float2bfloat16(c > 0.f ? __bfloat162float(g[i]) / c : 0.f);
}

// ------------------------------------------------------------------------------------------- host side
struct Layer {
  int cin, cout;
  size_t off;  // offset of W in the parameter arrays; the cout biases follow W
  size_t nw() const { return (size_t)cout * 9 * cin; }
};

struct Net {
  int device = 0;
  std::vector<Layer> L;
  size_t nparam = 0;
  float* w = nullptr;  // FP32 master parameters
  float* g = nullptr;  // gradients
  float* m = nullptr;  // AdamW moments
  float* v = nullptr;
  bf16* wb = nullptr;  // BF16 copy of the parameters (the forward pass reads weights from here, biases from w)
  bf16* wt = nullptr;  // flipped weights of one layer (data gradient)
  int step = 0;
  cudaStream_t st = nullptr;     // the net's own stream (training, calls without a stream)
  cudaEvent_t ws_done = nullptr; // recorded after every use of the workspace, on the stream of that use
  size_t ws_bytes = 0;
  char* ws = nullptr;            // activation (and gradient) workspace
  float* stats = nullptr;        // loss sum, valid count (loss kernel), valid count (count kernel)
  std::string err;
};

}  // namespace ps_cnn

struct ps_net {
  ps_cnn::Net n;
};

namespace ps_cnn {
namespace {

// (cin, cout) of the 12 convolutions, in parameter order.
const int kLayers[12][2] = {{48, 32}, {32, 32}, {32, 64}, {64, 64}, {64, 96}, {96, 96}, {96, 128}, {128, 128},
                            {224, 96}, {160, 64}, {96, 32}, {32, 8}};
enum { E0A, E0B, E1A, E1B, E2A, E2B, E3A, E3B, D2, D1, D0, HEAD };

inline unsigned blocks(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }
// Pixels per CTA of the weight gradient: at least `min_chunk`, a multiple of 16, and few enough chunks for grid.z.
inline int wgrad_chunk(long long P, int min_chunk) {
  long long c = (P + 65534) / 65535;
  c = (c + 15) / 16 * 16;
  return (int)(c > min_chunk ? c : min_chunk);
}

struct Fail {
  int code;
  std::string msg;
};
void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Fail{e == cudaErrorMemoryAllocation ? PS_ENOMEM : PS_ECUDA,
               std::string("CUDA: ") + what + ": " + cudaGetErrorString(e)};
  }
}

// Activation buffers of one pass at batch B and size H × W (multiples of 8), and their gradients for training.
struct Acts {
  bf16 *x, *a0, *s0, *p1, *a1, *s1, *p2, *a2, *s2, *p3, *a3, *b3, *c2, *d2, *c1, *d1, *c0, *d0;
  float* o;
  bf16 *g_o, *g_d0, *g_c0, *g_s0, *g_d1, *g_c1, *g_s1, *g_d2, *g_c2, *g_s2, *g_b3, *g_a3, *g_p3, *g_a2, *g_p2, *g_a1,
      *g_p1, *g_a0;
};

// Carves the workspace into the buffers of one pass on stream `st` (x and o only when the caller does not supply
// them).  The pass is ordered after the previous use of the workspace (possibly on another stream) through the
// ws_done event; growing the workspace waits for that use to finish on the host.  The caller records ws_done on `st`
// after its last launch (end_use).
void carve(Net& n, int B, int H, int W, Acts* A, bool grads, bool own_io, cudaStream_t st) {
  const long long P0 = (long long)B * H * W, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
  struct Item {
    void** p;
    size_t bytes;
  };
  std::vector<Item> it;
  Acts& a = *A;
  memset(&a, 0, sizeof a);
  auto add = [&](void* p, long long elems, size_t esz) { it.push_back({(void**)p, (size_t)elems * esz}); };
  if (own_io) {
    add(&a.x, P0 * 48, 2);
    add(&a.o, P0 * 8, 4);
  }
  add(&a.a0, P0 * 32, 2);
  add(&a.s0, P0 * 32, 2);
  add(&a.p1, P1 * 32, 2);
  add(&a.a1, P1 * 64, 2);
  add(&a.s1, P1 * 64, 2);
  add(&a.p2, P2 * 64, 2);
  add(&a.a2, P2 * 96, 2);
  add(&a.s2, P2 * 96, 2);
  add(&a.p3, P3 * 96, 2);
  add(&a.a3, P3 * 128, 2);
  add(&a.b3, P3 * 128, 2);
  if (grads) add(&a.c2, P2 * 224, 2);
  add(&a.d2, P2 * 96, 2);
  if (grads) add(&a.c1, P1 * 160, 2);
  add(&a.d1, P1 * 64, 2);
  if (grads) add(&a.c0, P0 * 96, 2);
  add(&a.d0, P0 * 32, 2);
  if (grads) {
    add(&a.g_o, P0 * 8, 2);
    add(&a.g_d0, P0 * 32, 2);
    add(&a.g_c0, P0 * 96, 2);
    add(&a.g_s0, P0 * 32, 2);
    add(&a.g_d1, P1 * 64, 2);
    add(&a.g_c1, P1 * 160, 2);
    add(&a.g_s1, P1 * 64, 2);
    add(&a.g_d2, P2 * 96, 2);
    add(&a.g_c2, P2 * 224, 2);
    add(&a.g_s2, P2 * 96, 2);
    add(&a.g_b3, P3 * 128, 2);
    add(&a.g_a3, P3 * 128, 2);
    add(&a.g_p3, P3 * 96, 2);
    add(&a.g_a2, P2 * 96, 2);
    add(&a.g_p2, P2 * 64, 2);
    add(&a.g_a1, P1 * 64, 2);
    add(&a.g_p1, P1 * 32, 2);
    add(&a.g_a0, P0 * 32, 2);
  }
  size_t total = 0;
  for (auto& i : it) total += (i.bytes + 255) & ~(size_t)255;
  if (total > n.ws_bytes) {
    ck(cudaEventSynchronize(n.ws_done), "wait for the workspace");
    if (n.ws) cudaFree(n.ws);
    n.ws = nullptr;
    n.ws_bytes = 0;
    ck(cudaMalloc(&n.ws, total), "cudaMalloc workspace");
    n.ws_bytes = total;
  }
  ck(cudaStreamWaitEvent(st, n.ws_done, 0), "order after the previous workspace use");
  size_t o = 0;
  for (auto& i : it) {
    *i.p = n.ws + o;
    o += (i.bytes + 255) & ~(size_t)255;
  }
}

void end_use(Net& n, cudaStream_t st) { ck(cudaEventRecord(n.ws_done, st), "record workspace use"); }

template <int BN>
void conv2_launch(const ConvArgs& a, cudaStream_t st) {
  constexpr size_t smem = conv2_smem<BN>();
  // opt-in to more than 48 KB of dynamic shared memory (per device; cheap, so on every launch)
  ck(cudaFuncSetAttribute(k_conv2<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "conv smem");
  const long long tiles = (long long)a.B * ((a.H + HT_H - 1) / HT_H) * ((a.W + HT_W - 1) / HT_W);
  dim3 g((unsigned)tiles, (unsigned)((a.cout + BN - 1) / BN));
  k_conv2<BN><<<g, 256, smem, st>>>(a);
}

template <int N>
void conv5_launch(const ConvArgs& a, cudaStream_t st) {
  constexpr size_t smem = Conv5Cfg<N>::smem;
  static_assert(smem <= 227 * 1024, "tcgen05 convolution tile exceeds shared memory");
  ck(cudaFuncSetAttribute(k_conv5<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "conv smem");
  constexpr int R = Conv5Cfg<N>::R;
  const long long ctas = (long long)a.B * ((a.H + R - 1) / R) * ((a.W + T5_PX - 1) / T5_PX);
  k_conv5<N><<<(unsigned)ctas, 128, smem, st>>>(a);
}

// 0: tcgen05 for cout in {64, 96, 128} (on B200 the 128 × 32 tile of cout = 32 is faster on mma.sync), 1: mma.sync
// only, 2: tcgen05 for every cout in {32, 64, 96, 128}
int g_conv_path = 0;

// cout in {32, 64, 96, 128}: tcgen05 (k_conv5); otherwise mma.sync (k_conv2) with the output-channel tile matched to
// cout (cout > 128 in two tiles: 224 -> 112, 160 -> 80).
void conv_launch(const ConvArgs& a, cudaStream_t st) {
  if (g_conv_path == 2 || (g_conv_path == 0 && a.cout >= 64)) switch (a.cout) {
      case 32: return conv5_launch<32>(a, st);
      case 64: return conv5_launch<64>(a, st);
      case 96: return conv5_launch<96>(a, st);
      case 128: return conv5_launch<128>(a, st);
      default: break;
    }
  switch (a.cout) {
    case 8: return conv2_launch<8>(a, st);
    case 16: return conv2_launch<16>(a, st);
    case 32: return conv2_launch<32>(a, st);
    case 48: return conv2_launch<48>(a, st);
    case 64: return conv2_launch<64>(a, st);
    case 96: return conv2_launch<96>(a, st);
    case 128: return conv2_launch<128>(a, st);
    case 160: return conv2_launch<80>(a, st);
    case 224: return conv2_launch<112>(a, st);
    default: break;
  }
  if (a.cout % 32 == 0) return conv2_launch<32>(a, st);
  return conv2_launch<8>(a, st);
}

// Layer li on x (channel stride xs), bias + optional ReLU; bf16 and/or f32 output.
void conv(Net& n, cudaStream_t st, int li, const bf16* x, int xs, bf16* y, float* yf, int B, int H, int W, int relu) {
  const Layer& l = n.L[li];
  ConvArgs a{};
  a.x = x;
  a.w = n.wb + l.off;
  a.bias = n.w + l.off + l.nw();
  a.y = y;
  a.yf = yf;
  a.B = B;
  a.H = H;
  a.W = W;
  a.cin = l.cin;
  a.cin_stride = xs;
  a.cin_off = 0;
  a.cout = l.cout;
  a.relu = relu;
  conv_launch(a, st);
}

// Layer li reading the virtual concatenation [up2(lo) (clo channels), skip (cskip channels)].
void conv_cat(Net& n, cudaStream_t st, int li, const bf16* lo, int clo, const bf16* skip, int cskip, bf16* y, int B,
              int H, int W) {
  const Layer& l = n.L[li];
  ConvArgs a{};
  memset(&a, 0, sizeof a);
  a.x = lo;
  a.w = n.wb + l.off;
  a.bias = n.w + l.off + l.nw();
  a.y = y;
  a.B = B;
  a.H = H;
  a.W = W;
  a.cin = l.cin;
  a.cin_stride = clo;
  a.cout = l.cout;
  a.relu = 1;
  a.x2 = skip;
  a.split = clo;
  a.x2_stride = cskip;
  conv_launch(a, st);
}

void forward(Net& n, const Acts& a, int B, int H, int W, cudaStream_t st) {
  const long long P0 = (long long)B * H * W, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
  const int H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
  conv(n, st, E0A, a.x, 48, a.a0, nullptr, B, H, W, 1);
  conv(n, st, E0B, a.a0, 32, a.s0, nullptr, B, H, W, 1);
  k_pool_fwd<<<blocks(P1 * 4), 256, 0, st>>>(a.s0, a.p1, B, H, W, 32);
  conv(n, st, E1A, a.p1, 32, a.a1, nullptr, B, H1, W1, 1);
  conv(n, st, E1B, a.a1, 64, a.s1, nullptr, B, H1, W1, 1);
  k_pool_fwd<<<blocks(P2 * 8), 256, 0, st>>>(a.s1, a.p2, B, H1, W1, 64);
  conv(n, st, E2A, a.p2, 64, a.a2, nullptr, B, H2, W2, 1);
  conv(n, st, E2B, a.a2, 96, a.s2, nullptr, B, H2, W2, 1);
  k_pool_fwd<<<blocks(P3 * 12), 256, 0, st>>>(a.s2, a.p3, B, H2, W2, 96);
  conv(n, st, E3A, a.p3, 96, a.a3, nullptr, B, H3, W3, 1);
  conv(n, st, E3B, a.a3, 128, a.b3, nullptr, B, H3, W3, 1);
  if (a.c2) {  // training: the concatenations are materialised (the backward pass reads them)
    k_up_fwd<<<blocks(P2 * 128), 256, 0, st>>>(a.b3, a.c2, B, H2, W2, 128, 224);
    k_copy_ch<<<blocks(P2 * 96), 256, 0, st>>>(a.s2, 96, 0, a.c2, 224, 128, 96, P2, 0);
    conv(n, st, D2, a.c2, 224, a.d2, nullptr, B, H2, W2, 1);
    k_up_fwd<<<blocks(P1 * 96), 256, 0, st>>>(a.d2, a.c1, B, H1, W1, 96, 160);
    k_copy_ch<<<blocks(P1 * 64), 256, 0, st>>>(a.s1, 64, 0, a.c1, 160, 96, 64, P1, 0);
    conv(n, st, D1, a.c1, 160, a.d1, nullptr, B, H1, W1, 1);
    k_up_fwd<<<blocks(P0 * 64), 256, 0, st>>>(a.d1, a.c0, B, H, W, 64, 96);
    k_copy_ch<<<blocks(P0 * 32), 256, 0, st>>>(a.s0, 32, 0, a.c0, 96, 64, 32, P0, 0);
    conv(n, st, D0, a.c0, 96, a.d0, nullptr, B, H, W, 1);
  } else {  // inference: upsampling and concatenation happen in the convolution's input loader
    conv_cat(n, st, D2, a.b3, 128, a.s2, 96, a.d2, B, H2, W2);
    conv_cat(n, st, D1, a.d2, 96, a.s1, 64, a.d1, B, H1, W1);
    conv_cat(n, st, D0, a.d1, 64, a.s0, 32, a.d0, B, H, W);
  }
  conv(n, st, HEAD, a.d0, 32, nullptr, a.o, B, H, W, 0);
  ck(cudaGetLastError(), "network forward");
}

// Backward of layer li: dW += Σ_p dY ⊗ im2col(X), db += Σ_p dY, and (dx != null) dX = conv(dY, flipped W).  dy is the
// gradient at the layer's pre-activation (already ReLU-masked).
void conv_bwd(Net& n, cudaStream_t st, int li, const bf16* dy, const bf16* x, int xs, bf16* dx, int B, int H, int W) {
  const Layer& l = n.L[li];
  const long long P = (long long)B * H * W;
  WgradArgs wa;
  wa.dy = dy;
  wa.x = x;
  wa.dw = n.g + l.off;
  wa.B = B;
  wa.H = H;
  wa.W = W;
  wa.cin = l.cin;
  wa.cin_stride = xs;
  wa.cin_off = 0;
  wa.cout = l.cout;
  wa.pix_per_cta = wgrad_chunk(P, 4096);
  dim3 g((unsigned)((l.cout + CM - 1) / CM), (unsigned)((9 * l.cin + CN - 1) / CN),
         (unsigned)((P + wa.pix_per_cta - 1) / wa.pix_per_cta));
  k_conv_wgrad<<<g, 128, 0, st>>>(wa);
  k_bias_grad<<<256, 256 / l.cout * l.cout, 0, st>>>(dy, n.g + l.off + l.nw(), P, l.cout);
  if (dx) {
    k_flip_weights<<<blocks((long long)l.nw()), 256, 0, st>>>(n.wb + l.off, n.wt, l.cout, l.cin);
    ConvArgs a{};
    a.x = dy;
    a.w = n.wt;
    a.bias = nullptr;
    a.y = dx;
    a.yf = nullptr;
    a.B = B;
    a.H = H;
    a.W = W;
    a.cin = l.cout;
    a.cin_stride = l.cout;
    a.cin_off = 0;
    a.cout = l.cin;
    a.relu = 0;
    conv_launch(a, st);
  }
}

void relu_bwd(bf16* dy, const bf16* y, long long cnt, cudaStream_t st) {
  k_relu_bwd<<<blocks(cnt), 256, 0, st>>>(dy, y, cnt);
}

void backward(Net& n, const Acts& a, int B, int H, int W, cudaStream_t st) {
  const long long P0 = (long long)B * H * W, P1 = P0 / 4, P2 = P0 / 16, P3 = P0 / 64;
  const int H1 = H / 2, W1 = W / 2, H2 = H / 4, W2 = W / 4, H3 = H / 8, W3 = W / 8;
  conv_bwd(n, st, HEAD, a.g_o, a.d0, 32, a.g_d0, B, H, W);
  relu_bwd(a.g_d0, a.d0, P0 * 32, st);
  conv_bwd(n, st, D0, a.g_d0, a.c0, 96, a.g_c0, B, H, W);
  // c0 = up(d1) ++ s0
  k_up_bwd<<<blocks(P1 * 64), 256, 0, st>>>(a.g_c0, a.g_d1, B, H, W, 64, 96);
  k_copy_ch<<<blocks(P0 * 32), 256, 0, st>>>(a.g_c0, 96, 64, a.g_s0, 32, 0, 32, P0, 0);
  relu_bwd(a.g_d1, a.d1, P1 * 64, st);
  conv_bwd(n, st, D1, a.g_d1, a.c1, 160, a.g_c1, B, H1, W1);
  // c1 = up(d2) ++ s1
  k_up_bwd<<<blocks(P2 * 96), 256, 0, st>>>(a.g_c1, a.g_d2, B, H1, W1, 96, 160);
  k_copy_ch<<<blocks(P1 * 64), 256, 0, st>>>(a.g_c1, 160, 96, a.g_s1, 64, 0, 64, P1, 0);
  relu_bwd(a.g_d2, a.d2, P2 * 96, st);
  conv_bwd(n, st, D2, a.g_d2, a.c2, 224, a.g_c2, B, H2, W2);
  // c2 = up(b3) ++ s2
  k_up_bwd<<<blocks(P3 * 128), 256, 0, st>>>(a.g_c2, a.g_b3, B, H2, W2, 128, 224);
  k_copy_ch<<<blocks(P2 * 96), 256, 0, st>>>(a.g_c2, 224, 128, a.g_s2, 96, 0, 96, P2, 0);
  // level 3
  relu_bwd(a.g_b3, a.b3, P3 * 128, st);
  conv_bwd(n, st, E3B, a.g_b3, a.a3, 128, a.g_a3, B, H3, W3);
  relu_bwd(a.g_a3, a.a3, P3 * 128, st);
  conv_bwd(n, st, E3A, a.g_a3, a.p3, 96, a.g_p3, B, H3, W3);
  k_pool_bwd<<<blocks(P2 * 96), 256, 0, st>>>(a.g_p3, a.g_s2, B, H2, W2, 96, 1);
  // level 2
  relu_bwd(a.g_s2, a.s2, P2 * 96, st);
  conv_bwd(n, st, E2B, a.g_s2, a.a2, 96, a.g_a2, B, H2, W2);
  relu_bwd(a.g_a2, a.a2, P2 * 96, st);
  conv_bwd(n, st, E2A, a.g_a2, a.p2, 64, a.g_p2, B, H2, W2);
  k_pool_bwd<<<blocks(P1 * 64), 256, 0, st>>>(a.g_p2, a.g_s1, B, H1, W1, 64, 1);
  // level 1
  relu_bwd(a.g_s1, a.s1, P1 * 64, st);
  conv_bwd(n, st, E1B, a.g_s1, a.a1, 64, a.g_a1, B, H1, W1);
  relu_bwd(a.g_a1, a.a1, P1 * 64, st);
  conv_bwd(n, st, E1A, a.g_a1, a.p1, 32, a.g_p1, B, H1, W1);
  k_pool_bwd<<<blocks(P0 * 32), 256, 0, st>>>(a.g_p1, a.g_s0, B, H, W, 32, 1);
  // level 0
  relu_bwd(a.g_s0, a.s0, P0 * 32, st);
  conv_bwd(n, st, E0B, a.g_s0, a.a0, 32, a.g_a0, B, H, W);
  relu_bwd(a.g_a0, a.a0, P0 * 32, st);
  conv_bwd(n, st, E0A, a.g_a0, a.x, 48, nullptr, B, H, W);
  ck(cudaGetLastError(), "network backward");
}

// splitmix64 -> uniform in [-1, 1)
inline double urand(uint64_t& s) {
  s += 0x9e3779b97f4a7c15ULL;
  uint64_t z = s;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return (double)(z >> 11) / (double)(1ULL << 53) * 2.0 - 1.0;
}

template <typename F>
int guard(Net& n, F&& f) {
  try {
    ck(cudaSetDevice(n.device), "cudaSetDevice");
    f();
    n.err.clear();
    return PS_OK;
  } catch (const Fail& e) {
    n.err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    n.err = "host allocation failed";
    return PS_ENOMEM;
  }
}

bool shape_ok(uint32_t B, uint32_t H, uint32_t W) {
  return B >= 1 && H >= 8 && W >= 8 && H % 8 == 0 && W % 8 == 0 && (uint64_t)B * H * W <= (1ull << 31);
}

void upload_params(Net& n, const float* host) {
  ck(cudaMemcpy(n.w, host, n.nparam * 4, cudaMemcpyHostToDevice), "upload parameters");
  std::vector<bf16> hb(n.nparam);
  for (size_t i = 0; i < n.nparam; ++i) hb[i] = __float2bfloat16(host[i]);
  ck(cudaMemcpy(n.wb, hb.data(), n.nparam * 2, cudaMemcpyHostToDevice), "upload parameters");
}

}  // namespace

// Forward of one batch on `st` (runtime entry: the caller orders its producer and consumer on the same stream).
int forward_on_stream(ps_net* pn, const void* in, int B, int H, int W, float* out, cudaStream_t st, std::string* err) {
  if (!pn || !in || !out || !shape_ok(B, H, W)) return PS_EINVAL;
  Net& n = pn->n;
  const int rc = guard(n, [&] {
    Acts a;
    carve(n, B, H, W, &a, false, false, st);
    a.x = (bf16*)in;
    a.o = out;
    forward(n, a, B, H, W, st);
    end_use(n, st);
  });
  if (rc != PS_OK && err) *err = n.err;
  return rc;
}

int conv_health(std::string* err) {
  unsigned c = 0;
  if (cudaMemcpyFromSymbol(&c, g_conv5_timeouts, sizeof c) != cudaSuccess) {
    cudaGetLastError();
    if (err) *err = "cannot read the tensor-core convolution status";
    return PS_ECUDA;
  }
  if (c) {
    if (err) *err = std::to_string(c) + " tensor-core convolution wait(s) expired: network outputs are invalid";
    return PS_ETIMEOUT;
  }
  return PS_OK;
}

cudaError_t launch_decode(const float* o, int Wp, int H, int W, float4* planes, float* conf, float inv_near,
                          float inv_far, float thr, const float* k, unsigned long long* count, cudaStream_t st) {
  dim3 b(32, 8), g((W + 31) / 32, (H + 7) / 8);
  k_decode<<<g, b, 0, st>>>(o, Wp, H, W, planes, conf, inv_near, inv_far, thr, k[0], k[1], k[2], k[3], count);
  return cudaGetLastError();
}

}  // namespace ps_cnn

using namespace ps_cnn;

extern "C" {

int ps_net_create(int device, uint64_t seed, ps_net** out) {
  if (!out) return PS_EINVAL;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return PS_ENODEV;
  }
  ps_net* pn = new (std::nothrow) ps_net();
  if (!pn) return PS_ENOMEM;
  Net& n = pn->n;
  n.device = device;
  const int rc = guard(n, [&] {
    size_t off = 0, maxw = 0;
    for (auto& l : kLayers) {
      Layer L{l[0], l[1], off};
      n.L.push_back(L);
      off += L.nw() + (size_t)L.cout;
      maxw = L.nw() > maxw ? L.nw() : maxw;
    }
    n.nparam = off;
    ck(cudaStreamCreateWithFlags(&n.st, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreateWithFlags(&n.ws_done, cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaMalloc(&n.w, off * 4), "cudaMalloc");
    ck(cudaMalloc(&n.g, off * 4), "cudaMalloc");
    ck(cudaMalloc(&n.m, off * 4), "cudaMalloc");
    ck(cudaMalloc(&n.v, off * 4), "cudaMalloc");
    ck(cudaMalloc(&n.wb, off * 2), "cudaMalloc");
    ck(cudaMalloc(&n.wt, maxw * 2), "cudaMalloc");
    ck(cudaMalloc(&n.stats, 64), "cudaMalloc");
    // He-uniform weights (fan-in 9·cin; the head ×0.1), zero biases; input channels 33..47 carry zeros and get zero
    // weights
    std::vector<float> h(off, 0.f);
    uint64_t s = seed;
    for (size_t li = 0; li < n.L.size(); ++li) {
      const Layer& L = n.L[li];
      const double bound = sqrt(6.0 / (9.0 * L.cin)) * (li == HEAD ? 0.1 : 1.0);
      for (size_t i = 0; i < L.nw(); ++i) {
        const int ci = (int)(i % L.cin);
        h[L.off + i] = (li == E0A && ci >= 1 + PS_SWEEP_PLANES) ? 0.f : (float)(bound * urand(s));
      }
    }
    upload_params(n, h.data());
    ck(cudaMemset(n.m, 0, off * 4), "cudaMemset");
    ck(cudaMemset(n.v, 0, off * 4), "cudaMemset");
  });
  if (rc != PS_OK) {
    ps_net_destroy(pn);
    return rc;
  }
  *out = pn;
  return PS_OK;
}

void ps_net_destroy(ps_net* pn) {
  if (!pn) return;
  Net& n = pn->n;
  if (cudaSetDevice(n.device) == cudaSuccess) {
    if (n.st) cudaStreamSynchronize(n.st);
    if (n.ws_done) cudaEventSynchronize(n.ws_done);  // a use on a caller's stream (that stream may be gone by now)
    cudaFree(n.w);
    cudaFree(n.g);
    cudaFree(n.m);
    cudaFree(n.v);
    cudaFree(n.wb);
    cudaFree(n.wt);
    cudaFree(n.ws);
    cudaFree(n.stats);
    if (n.st) cudaStreamDestroy(n.st);
    if (n.ws_done) cudaEventDestroy(n.ws_done);
  }
  cudaGetLastError();
  delete pn;
}

const char* ps_net_last_error(const ps_net* pn) { return pn ? pn->n.err.c_str() : "net is NULL"; }

int ps_net_set_conv_path(int path) {
  if (path < 0 || path > 2) return PS_EINVAL;
  g_conv_path = path;
  return PS_OK;
}

int ps_net_test_stall_convolutions(int device, int on) {
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return PS_ENODEV;
  }
  const int v = on ? 1 : 0;
  if (cudaMemcpyToSymbol(g_conv5_stall, &v, sizeof v) != cudaSuccess) {
    cudaGetLastError();
    return PS_ECUDA;
  }
  return PS_OK;
}

int ps_net_conv_timeouts(int device, uint32_t* count, int reset) {
  if (!count) return PS_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return PS_ENODEV;
  }
  unsigned c = 0;
  if (cudaMemcpyFromSymbol(&c, g_conv5_timeouts, sizeof c) != cudaSuccess) {
    cudaGetLastError();
    return PS_ECUDA;
  }
  *count = c;
  if (reset) {
    const unsigned z = 0;
    if (cudaMemcpyToSymbol(g_conv5_timeouts, &z, sizeof z) != cudaSuccess) {
      cudaGetLastError();
      return PS_ECUDA;
    }
  }
  return PS_OK;
}
uint64_t ps_net_num_params(const ps_net* pn) { return pn ? (uint64_t)pn->n.nparam : 0; }
uint32_t ps_net_step(const ps_net* pn) { return pn ? (uint32_t)pn->n.step : 0; }

int ps_net_get_params(ps_net* pn, float* host) {
  if (!pn || !host) return PS_EINVAL;
  return guard(pn->n, [&] {
    ck(cudaStreamSynchronize(pn->n.st), "sync");
    ck(cudaMemcpy(host, pn->n.w, pn->n.nparam * 4, cudaMemcpyDeviceToHost), "download parameters");
  });
}

int ps_net_set_params(ps_net* pn, const float* host) {
  if (!pn || !host) return PS_EINVAL;
  return guard(pn->n, [&] {
    ck(cudaStreamSynchronize(pn->n.st), "sync");
    ck(cudaEventSynchronize(pn->n.ws_done), "sync");  // parameters are read by passes on callers' streams too
    upload_params(pn->n, host);
  });
}

int ps_net_train_step(ps_net* pn, const void* input, const float* labels, uint32_t B, uint32_t H, uint32_t W,
                      float depth_min, float depth_max, float lr, float weight_decay, float* loss_out,
                      float* grad_out) {
  if (!pn || !input || !labels || !shape_ok(B, H, W) || !(depth_min > 0.f) || !(depth_max > depth_min) ||
      !(lr >= 0.f))
    return PS_EINVAL;
  return guard(pn->n, [&] {
    Net& n = pn->n;
    cudaStream_t st = n.st;
    Acts a;
    carve(n, B, H, W, &a, true, false, st);
    a.x = (bf16*)input;
    const long long P0 = (long long)B * H * W;
    ck(cudaMallocAsync((void**)&a.o, P0 * 8 * 4, st), "cudaMallocAsync");
    forward(n, a, B, H, W, st);
    ck(cudaMemsetAsync(n.stats, 0, 64, st), "cudaMemset");
    ck(cudaMemsetAsync(n.g, 0, n.nparam * 4, st), "cudaMemset");
    k_count_valid<<<blocks(P0), 256, 0, st>>>(labels, P0, n.stats + 2);
    k_loss<<<blocks(P0), 256, 0, st>>>(a.o, labels, a.g_o, n.stats, P0, 1.f, 1.f / depth_min, 1.f / depth_max);
    k_scale_grad<<<blocks(P0 * 8), 256, 0, st>>>(a.g_o, P0 * 8, n.stats + 2);
    backward(n, a, B, H, W, st);
    end_use(n, st);
    ck(cudaFreeAsync(a.o, st), "cudaFreeAsync");
    if (grad_out) ck(cudaMemcpyAsync(grad_out, n.g, n.nparam * 4, cudaMemcpyDeviceToHost, st), "gradients");
    if (lr > 0.f) {
      n.step++;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.f - powf(b1, (float)n.step), c2 = 1.f - powf(b2, (float)n.step);
      for (auto& L : n.L) {  // weights with decoupled weight decay, biases without
        k_adamw<<<blocks((long long)L.nw()), 256, 0, st>>>(n.w + L.off, n.g + L.off, n.m + L.off, n.v + L.off,
                                                            n.wb + L.off, (long long)L.nw(), lr, b1, b2, 1e-8f,
                                                            weight_decay, c1, c2);
        const size_t bo = L.off + L.nw();
        k_adamw<<<blocks(L.cout), 256, 0, st>>>(n.w + bo, n.g + bo, n.m + bo, n.v + bo, n.wb + bo, L.cout, lr, b1, b2,
                                                 1e-8f, 0.f, c1, c2);
      }
    }
    ck(cudaGetLastError(), "training step");
    float sv[2] = {0.f, 0.f};
    ck(cudaMemcpyAsync(sv, n.stats, 8, cudaMemcpyDeviceToHost, st), "loss");
    ck(cudaStreamSynchronize(st), "sync");
    if (loss_out) *loss_out = sv[1] > 0.f ? sv[0] / sv[1] : 0.f;
    std::string e;
    const int h = conv_health(&e);
    if (h != PS_OK) throw Fail{h, e};
  });
}

int ps_net_forward(ps_net* pn, const void* input, uint32_t B, uint32_t H, uint32_t W, float* out, void* stream) {
  if (!pn || !input || !out || !shape_ok(B, H, W)) return PS_EINVAL;
  return guard(pn->n, [&] {
    Net& n = pn->n;
    cudaStream_t st = stream ? (cudaStream_t)stream : n.st;
    Acts a;
    carve(n, B, H, W, &a, false, false, st);
    a.x = (bf16*)input;
    a.o = out;
    forward(n, a, B, H, W, st);
    end_use(n, st);
    if (!stream) {
      ck(cudaStreamSynchronize(st), "sync");
      std::string e;
      const int h = conv_health(&e);
      if (h != PS_OK) throw Fail{h, e};
    }
  });
}

int ps_net_conv_check(int device, const uint16_t* x, const float* w, const uint16_t* dy, uint32_t B, uint32_t H,
                      uint32_t W, uint32_t cin, uint32_t cout, float* y, float* dx, float* dw) {
  if (!x || !w || !dy || !y || !dx || !dw || cin < 8 || cin % 8 || cout < 8 || cout % 8 || !shape_ok(B, 8, 8) ||
      H < 1 || W < 1 || (uint64_t)B * H * W > (1u << 24))
    return PS_EINVAL;
  Net n;
  n.device = device;
  struct Bufs {
    bf16 *x = nullptr, *dy = nullptr, *wb = nullptr, *wt = nullptr;
    float *y = nullptr, *dx = nullptr, *dw = nullptr;
    ~Bufs() {
      cudaFree(x);
      cudaFree(dy);
      cudaFree(wb);
      cudaFree(wt);
      cudaFree(y);
      cudaFree(dx);
      cudaFree(dw);
    }
  };
  return guard(n, [&] {
    Bufs b;
    const long long P = (long long)B * H * W;
    const size_t nw = (size_t)cout * 9 * cin;
    ck(cudaMalloc(&b.x, P * cin * 2), "cudaMalloc");
    ck(cudaMalloc(&b.dy, P * cout * 2), "cudaMalloc");
    ck(cudaMalloc(&b.wb, nw * 2), "cudaMalloc");
    ck(cudaMalloc(&b.wt, nw * 2), "cudaMalloc");
    ck(cudaMalloc(&b.y, P * cout * 4), "cudaMalloc");
    ck(cudaMalloc(&b.dx, P * cin * 4), "cudaMalloc");
    ck(cudaMalloc(&b.dw, nw * 4), "cudaMalloc");
    std::vector<bf16> hw(nw);
    for (size_t i = 0; i < nw; ++i) hw[i] = __float2bfloat16(w[i]);
    ck(cudaMemcpy(b.x, x, P * cin * 2, cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(b.dy, dy, P * cout * 2, cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(b.wb, hw.data(), nw * 2, cudaMemcpyHostToDevice), "upload");
    ck(cudaMemset(b.dw, 0, nw * 4), "cudaMemset");
    ConvArgs a{};
    a.x = b.x;
    a.w = b.wb;
    a.bias = nullptr;
    a.y = nullptr;
    a.yf = b.y;
    a.B = (int)B;
    a.H = (int)H;
    a.W = (int)W;
    a.cin = (int)cin;
    a.cin_stride = (int)cin;
    a.cin_off = 0;
    a.cout = (int)cout;
    a.relu = 0;
    conv_launch(a, 0);
    k_flip_weights<<<blocks((long long)nw), 256>>>(b.wb, b.wt, (int)cout, (int)cin);
    ConvArgs d = a;
    d.x = b.dy;
    d.w = b.wt;
    d.cin = (int)cout;
    d.cin_stride = (int)cout;
    d.cout = (int)cin;
    d.yf = b.dx;
    conv_launch(d, 0);
    WgradArgs wa;
    wa.dy = b.dy;
    wa.x = b.x;
    wa.dw = b.dw;
    wa.B = (int)B;
    wa.H = (int)H;
    wa.W = (int)W;
    wa.cin = (int)cin;
    wa.cin_stride = (int)cin;
    wa.cin_off = 0;
    wa.cout = (int)cout;
    wa.pix_per_cta = wgrad_chunk(P, 256);
    dim3 g((unsigned)((cout + CM - 1) / CM), (unsigned)((9 * cin + CN - 1) / CN),
           (unsigned)((P + wa.pix_per_cta - 1) / wa.pix_per_cta));
    k_conv_wgrad<<<g, 128>>>(wa);
    ck(cudaGetLastError(), "convolution kernels");
    ck(cudaDeviceSynchronize(), "sync");
    ck(cudaMemcpy(y, b.y, P * cout * 4, cudaMemcpyDeviceToHost), "download");
    ck(cudaMemcpy(dx, b.dx, P * cin * 4, cudaMemcpyDeviceToHost), "download");
    ck(cudaMemcpy(dw, b.dw, nw * 4, cudaMemcpyDeviceToHost), "download");
  });
}

}  // extern "C"
