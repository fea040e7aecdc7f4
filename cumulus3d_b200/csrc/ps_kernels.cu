// PatchStereo kernels for sm_100a.
//
// Compiled three times into libpatchstereo.so:
//   PS_FAST=0 (namespace ps_parity): --fmad=false, IEEE division and square root, the project's own exp/sincos
//            (ps_fmath.h) and fma only where written out.  Bitwise equal to the CPU oracle (oracle/ps_oracle.cpp),
//            which follows the same operation sequence.
//   PS_FAST=1 (namespace ps_fast):   --use_fast_math, hardware reciprocal / exp / rsqrt in the hot loops
//            ("the kernel may use approximate division and exponential", crates/dense/src/kernel.rs:73-74).
//   PS_CHECKED=1 (namespace ps_checked): the parity build plus bounds tests on every data-dependent index (tile,
//            staged box, source plane, state arrays, source view, snapshot); a failed test skips the access and
//            records the first violation in PsRun.fault (see PsCheckSite), which the runtime reports as PS_EFAULT.
//
// The rules are those of the reference kernel crates/cuda/src/kernels/patchmatch.cu (cited per function) and of
// crates/dense/src/kernel.rs:36-74.  The B200 layout differs from the reference:
//   * every image level is a normalised f32 plane with a PS_BORDER-pixel zero border, so a bilinear source tap is
//     four unconditional loads after a clamp (no per-texel bounds tests); optionally (PS_TUNE_TEX_GATHER) a gather
//     through a border-addressed texture fetches the same four texels with one instruction;
//   * a half-step CTA is 128 threads covering a 32 × 8 pixel tile; each warp takes 16 active columns of two
//     adjacent rows, so reference-tile reads of the two colour phases fall into disjoint shared-memory banks;
//   * the bilateral window weights of a pixel are computed once per half step and cached in shared memory (one
//     slot per thread and tap) and reused by all 9·N + 6·a NCC evaluations of that pixel;
//   * launches are flattened over the tiles of all views of a batch (no idle CTAs for ragged batches); the batch
//     table travels in the kernel parameters.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include "ps_fmath.h"
#include "ps_pairs.h"
#include "ps_types.h"

#ifndef PS_FAST
#define PS_FAST 0
#endif
#ifndef PS_CHECKED
#define PS_CHECKED 0
#endif
#if PS_FAST && PS_CHECKED
#error "the bounds-checked build uses the parity math"
#endif
#if PS_FAST
#define PS_NS ps_fast
#elif PS_CHECKED
#define PS_NS ps_checked
#else
#define PS_NS ps_parity
#endif

typedef unsigned long long u64;

namespace PS_NS {

// ------------------------------------------------------------------------------------------- bounds tests
// PS_IN(fault, site, idx, lo, hi): lo <= idx < hi.  In the checked build a failure records (site, idx) once per launch
// (the first failure wins) and the caller skips the access; in the other builds the test is absent (true, and the
// arguments are not evaluated).
#if PS_CHECKED
__device__ __noinline__ void chk_record(unsigned long long* fault, unsigned site, long long idx) {
  if (fault)
    atomicCAS(fault, 0ull, ((unsigned long long)site << 56) | ((unsigned long long)idx & 0x00FFFFFFFFFFFFFFull));
}
__device__ __forceinline__ bool chk_in(unsigned long long* fault, unsigned site, long long idx, long long lo,
                                       long long hi) {
  if (idx >= lo && idx < hi) return true;
  chk_record(fault, site, idx);
  return false;
}
#define PS_IN(fault, site, idx, lo, hi) chk_in((fault), (site), (long long)(idx), (long long)(lo), (long long)(hi))
#else
#define PS_IN(fault, site, idx, lo, hi) true
#endif

// ------------------------------------------------------------------------------------------- math policy
__device__ __forceinline__ float m_rcp(float x) {
#if PS_FAST
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
#else
  // Correctly rounded reciprocal (the oracle's IEEE 1/x): the hardware approximation rcp.approx (within 1 ulp)
  // refined by one Newton-Raphson correction on the exact FMA residual e = 1 - x*r, r' = r + r*e rounded once
  // (Markstein's FMA correction).  The result equals the round-to-nearest-even reciprocal for every x in
  // [2^-126, 2^126), checked exhaustively over all significands by k_rcp_check (ps_check_reciprocal); the kernels
  // only take reciprocals of projective depths above 1e-8.
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return fmaf(r, fmaf(-x, r, 1.0f), r);
#endif
}
__device__ __forceinline__ float m_exp(float x) {
#if PS_FAST
  return __expf(x);
#else
  return ps_expf(x);
#endif
}
__device__ __forceinline__ void m_sincos(float x, float* s, float* c) {
#if PS_FAST
  __sincosf(x, s, c);
#else
  ps_sincosf(x, s, c);
#endif
}
__device__ __forceinline__ float m_rsqrt(float x) {
#if PS_FAST
  return rsqrtf(x);
#else
  return 1.0f / sqrtf(x);
#endif
}

// ------------------------------------------------------------------------------------------- RNG (patchmatch.cu:112-125)
__device__ __forceinline__ u64 mix64(u64 z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
__device__ __forceinline__ float rnd(u64& s) {
  s += 0x9e3779b97f4a7c15ULL;
  u64 z = mix64(s);
  return ((float)(z >> 40) + 1.0f) * (1.0f / 16777216.0f);
}
__device__ __forceinline__ u64 rng_state(u64 seed, u64 key, int level, int run, int t, int half, u64 pixel) {
  u64 tag = ((u64)level << 48) ^ ((u64)run << 32) ^ ((u64)t << 16) ^ (u64)half;
  return mix64(seed ^ mix64(key ^ mix64(tag)) ^ pixel);
}

// ------------------------------------------------------------------------------------------- vectors (patchmatch.cu:128-133)
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 nrm3(float3 a) {
  float l = m_rsqrt(fmaxf(dot3(a, a), 1e-30f));
  return make_float3(a.x * l, a.y * l, a.z * l);
}
// patchmatch.cu:386
__device__ __forceinline__ float3 pixel_ray(const PsLevel& R, int x, int y) {
  return make_float3(((float)x - R.cx) / R.fx, ((float)y - R.cy) / R.fy, 1.0f);
}

// ------------------------------------------------------------------------------------------- source sample (patchmatch.cu:169-192)
// Bilinear value at (u, v), integer-centre convention, 0 outside the image.  The clamp to [-2, w] × [-2, h] keeps
// both taps of an out-of-image footprint inside the zero border, which reproduces the reference's "0 outside"
// without per-texel tests.
__device__ __forceinline__ int f2i_exact(float v) {
  // v is an integer in [-2^22, 2^22]: adding 1.5·2^23 puts it in the low mantissa bits (one FADD instead of the
  // quarter-rate F2I conversion).
  return __float_as_int(v + 12582912.0f) - 0x4B400000;
}
__device__ __forceinline__ float src_sample(const float* __restrict__ img, int pitch, float wf, float hf, float u,
                                            float v, unsigned long long* fault = nullptr) {
  float xf = floorf(u), yf = floorf(v);
  float ax = u - xf, ay = v - yf;
  float xc = fminf(fmaxf(xf, -2.0f), wf);
  float yc = fminf(fmaxf(yf, -2.0f), hf);
#if PS_CHECKED
  // the 2 × 2 footprint inside the bordered plane: columns [-PS_BORDER, pitch - PS_BORDER), rows [-PS_BORDER,
  // h + PS_BORDER)
  if (!PS_IN(fault, PS_SITE_PLANE, f2i_exact(xc), -PS_BORDER, pitch - PS_BORDER - 1) ||
      !PS_IN(fault, PS_SITE_PLANE, f2i_exact(yc), -PS_BORDER, (int)hf + PS_BORDER - 1))
    return 0.f;
#endif
  const float* p = img + f2i_exact(yc) * pitch + f2i_exact(xc);
  float p00 = __ldg(p), p10 = __ldg(p + 1), p01 = __ldg(p + pitch), p11 = __ldg(p + pitch + 1);
  float top = fmaf(ax, p10 - p00, p00);
  float bot = fmaf(ax, p11 - p01, p01);
  return fmaf(ay, bot - top, top);
}
// Same sample through the texture unit: a gather at the exact integer coordinate (x0, y0) selects the footprint
// (x0-1 .. x0, y0-1 .. y0), and the texel offset (+1, +1) of the tld4 instruction moves it onto (x0 .. x0+1,
// y0 .. y0+1), so the four texels come back without two coordinate additions per tap (border addressing gives 0
// outside the image).  The bilinear arithmetic is unchanged, so the result has the same bits as src_sample.
// Gather order: (T[x0,y1], T[x1,y1], T[x1,y0], T[x0,y0]).
__device__ __forceinline__ float4 gather_red_offset11(unsigned long long tex, float x, float y) {
  float4 q;
  asm("tld4.r.2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6}], {%7, %8};"
      : "=f"(q.x), "=f"(q.y), "=f"(q.z), "=f"(q.w)
      : "l"(tex), "f"(x), "f"(y), "r"(1), "r"(1));
  return q;
}
__device__ __forceinline__ float src_sample_tex(unsigned long long tex, float u, float v) {
  float xf = floorf(u), yf = floorf(v);
  float ax = u - xf, ay = v - yf;
  const float4 q = gather_red_offset11(tex, xf, yf);
  const float p00 = q.w, p10 = q.z, p01 = q.x, p11 = q.y;
  float top = fmaf(ax, p10 - p00, p00);
  float bot = fmaf(ax, p11 - p01, p01);
  return fmaf(ay, bot - top, top);
}

// ------------------------------------------------------------------------------------------- reference window
struct RefStats {
  float ic, W, mu, var;
};

// Tile-resident reference window of one pixel: t points at the pixel inside the shared tile (row pitch tw); wc is
// the thread's weight-cache slot (stride NT floats between taps).  Window sums are split by row parity: even rows
// (a = 0, 2, …) and odd rows (a = 1, 3, …) accumulate separately, in ascending row order, and the NCC uses
// even + odd.  With G = 2 lanes per pixel, lane g sums the rows of parity g and the two partial sums meet through
// one shuffle (pmask = the pair's lanes); with G = 1 one thread keeps both partial sums.
//
// Weight-cache layouts: per tap (a, b) one float per thread, stride NT between taps.  The legacy layout keeps row a at
// wc + a·wn·NT.  The row-pair layout (PW) used by the f32x2 tap loops puts the weights of rows 2p and 2p+1 of the
// same column next to each other (one 8-byte load per tap pair): wc + (p·wn + b)·2·NT + (a & 1) with wc = base +
// 2·thread, and the last row of an odd window at wl + b·NT.
struct RefWin {
  const float* t;
  int tw;
  float* wc;
  int g;
  unsigned pmask;
  float* wl;
#if PS_CHECKED
  const float* tbase;  // the tile and its size in floats
  int tn;
  unsigned long long* fault;
#endif
};

// Bounds of the tile a RefWin reads (checked build only).
__device__ __forceinline__ void refwin_bounds(RefWin& rw, const float* tile, int n, const PsRun& P) {
#if PS_CHECKED
  rw.tbase = tile;
  rw.tn = n;
  rw.fault = P.fault;
#endif
}
// Reference intensity at p inside the tile.
__device__ __forceinline__ float tile_at(const RefWin& rw, const float* p) {
#if PS_CHECKED
  if (!PS_IN(rw.fault, PS_SITE_TILE, p - rw.tbase, 0, rw.tn)) return 0.f;
#endif
  return *p;
}

// Row-parity partial sums -> total (even + odd; IEEE addition is commutative, so both lanes get the same bits).
template <int G>
__device__ __forceinline__ float pair_total(const RefWin& rw, const float* part) {
  if constexpr (G == 1) {
    return part[0] + part[1];
  } else {
    const float other = __shfl_xor_sync(rw.pmask, part[0], 1);
    return part[0] + other;
  }
}

// ref_stats (patchmatch.cu:199-223).  Weights w_k = exp(-(dx²+dy²)/(2σs²) - (Ic-Ik)²/(2σc²)); 0 outside the image.
template <int WR, int WS, bool CW, int NT, int G = 1, bool PW = false>
__device__ __forceinline__ RefStats ref_stats(const PsRun& P, const RefWin& rw) {
  const int wr = WR ? WR : P.wr, ws = WR ? WS : P.ws;
  const int wn = (2 * wr) / ws + 1;
  RefStats s;
  s.ic = tile_at(rw, rw.t);
  float W[2] = {0.f, 0.f}, S[2] = {0.f, 0.f}, SS[2] = {0.f, 0.f};
#pragma unroll 1
  for (int a = (G == 2 ? rw.g : 0); a < wn; a += G) {
    const int dy = -wr + a * ws;
    const int pa = G == 2 ? 0 : (a & 1);
    const float* trow = rw.t + dy * rw.tw;
    float* wrow;
    int wst = NT;
    if constexpr (PW) {
      if (a < (wn & ~1)) {
        wrow = rw.wc + (a >> 1) * wn * NT * 2 + (a & 1);
        wst = 2 * NT;
      } else {
        wrow = rw.wl;
      }
    } else {
      wrow = rw.wc + (G == 2 ? (a >> 1) : a) * wn * NT;
    }
    auto tap = [&](int b) {
      const int dx = -wr + b * ws;
      float ik = tile_at(rw, trow + dx);
      float d = s.ic - ik;
      float w = m_exp(-(float)(dx * dx + dy * dy) * P.inv2s - d * d * P.inv2c);
      if (CW) wrow[b * wst] = w;
      float wi = w * ik;
      W[pa] = W[pa] + w;
      S[pa] = S[pa] + wi;
      SS[pa] = fmaf(wi, ik, SS[pa]);
    };
    if constexpr (WR != 0) {
#pragma unroll
      for (int b = 0; b < (2 * WR) / WS + 1; ++b) tap(b);
    } else {
#pragma unroll 1
      for (int b = 0; b < wn; ++b) tap(b);
    }
  }
  s.W = pair_total<G>(rw, W);
  const float St = pair_total<G>(rw, S), SSt = pair_total<G>(rw, SS);
  s.mu = St / s.W;
  s.var = SSt / s.W - s.mu * s.mu;
  return s;
}

// Plane-induced homography H = A + b (nᵀK⁻¹)/δ (patchmatch.cu:225-242).
__device__ __forceinline__ bool homography(const PsLevel& R, const PsLPair& L, float x, float y, float4 h, float* H) {
  float ifx = 1.0f / R.fx, ify = 1.0f / R.fy;
  float3 n = make_float3(h.x, h.y, h.z);
  float3 ray = make_float3((x - R.cx) * ifx, (y - R.cy) * ify, 1.0f);
  float delta = h.w * dot3(n, ray);
  if (!(delta < -1e-12f)) return false;
  float id = 1.0f / delta;
  float u0 = n.x * ifx, u1 = n.y * ify;
  float u2 = n.z - u0 * R.cx - u1 * R.cy;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    float br = L.b[r] * id;
    H[r * 3 + 0] = L.A[r * 3 + 0] + br * u0;
    H[r * 3 + 1] = L.A[r * 3 + 1] + br * u1;
    H[r * 3 + 2] = L.A[r * 3 + 2] + br * u2;
  }
  return true;
}

// Cost 1 - ρ of the bilateral-weighted NCC (patchmatch.cu:245-290); 2 on failure.
// Parity operation sequence per tap (dx, dy), with sx = x+dx, sy = y+dy:
//   zz = fma(H6, sx, fma(H7, sy, H8)); if zz > 1e-8: s = sample(fma(H0,sx,fma(H1,sy,H2))·(1/zz), fma(H3,sx,fma(H4,sy,H5))·(1/zz))
//   ws = w·s; Ss += ws; SSs = fma(ws, s, SSs); IS = fma(ws, Ik, IS)
//
// Prologue (patchmatch.cu:251-262): the window centre must project in front of the source camera and inside the
// image, and the reference window must have variance; otherwise the cost is 2 and no window is evaluated.
__device__ __forceinline__ bool ncc_begin(const RefStats& rs, const PsLevel& S, const float* H, float fx, float fy) {
  const float z = fmaf(H[6], fx, fmaf(H[7], fy, H[8]));
  if (!(z > 1e-8f)) return false;
  const float iz = m_rcp(z);
  const float u = fmaf(H[0], fx, fmaf(H[1], fy, H[2])) * iz;
  const float v = fmaf(H[3], fx, fmaf(H[4], fy, H[5])) * iz;
  const float wf = (float)S.w, hf = (float)S.h;
  if (!(u >= 0.f && v >= 0.f && u <= wf - 1.0f && v <= hf - 1.0f)) return false;
  return !(rs.var < 1e-5f);
}
// Epilogue (patchmatch.cu:280-289) from the window totals.
__device__ __forceinline__ float ncc_finish(const RefStats& rs, float Sst, float SSst, float ISt) {
  float iW = 1.0f / rs.W;
  float mus = Sst * iW;
  float vars = SSst * iW - mus * mus;
  if (vars < 1e-5f) return 2.0f;
  float cov = ISt * iW - rs.mu * mus;
#if PS_FAST
  float c = 1.0f - cov * rsqrtf(rs.var * vars);
#else
  float c = 1.0f - cov / sqrtf(rs.var * vars);
#endif
  return fminf(fmaxf(c, 0.0f), 2.0f);
}

// Window sums over the taps (patchmatch.cu:263-279) and the cost; the prologue must have passed.
//
// A tap behind the source camera (zz <= 1e-8) samples 0.  The computed zz = fma(H6, sx, fma(H7, sy, H8)) is monotone
// in sx for a fixed row and, through the correctly rounded inner fma, monotone in sy for a fixed column (each step is
// a correctly rounded function of an affine expression, and rounding is monotone), so the smallest zz of the window
// is at one of its four corner taps.  When all four are in front, every tap is, and the taps run without the
// per-tap test and selects; otherwise a guarded loop handles each tap (the same bits either way).
template <int WR, int WS, bool CW, int NT, bool TEX, int G, bool PW = false>
__device__ __forceinline__ float ncc_window(const PsRun& P, const RefWin& rw, const RefStats& rs, const PsLevel& S,
                                            const float* H, int x, int y) {
  const int wr = WR ? WR : P.wr, ws = WR ? WS : P.ws;
  const int wn = (2 * wr) / ws + 1;
  const float fx = (float)x, fy = (float)y;
  const float wf = (float)S.w, hf = (float)S.h;
  const float* __restrict__ img = S.img;
  const unsigned long long tex = S.tex;
  const int pitch = S.pitch;
  float Ss[2] = {0.f, 0.f}, SSs[2] = {0.f, 0.f}, IS[2] = {0.f, 0.f};
  const float sx0 = fx + (float)(-wr), sx1 = fx + (float)wr;
  const float rz0 = fmaf(H[7], fy + (float)(-wr), H[8]), rz1 = fmaf(H[7], fy + (float)wr, H[8]);
  const bool all_front = fmaf(H[6], sx0, rz0) > 1e-8f && fmaf(H[6], sx1, rz0) > 1e-8f &&
                         fmaf(H[6], sx0, rz1) > 1e-8f && fmaf(H[6], sx1, rz1) > 1e-8f;
  auto sample = [&](float uf, float vf) {
    if constexpr (TEX) return src_sample_tex(tex, uf, vf);
    else return src_sample(img, pitch, wf, hf, uf, vf, P.fault);
  };
  auto accumulate = [&](int pa, float w, float sv, float ik) {
    const float wsv = w * sv;
    Ss[pa] = Ss[pa] + wsv;
    SSs[pa] = fmaf(wsv, sv, SSs[pa]);
    IS[pa] = fmaf(wsv, ik, IS[pa]);
  };
  // weights of row a start at wrow(a), stride wst(a) between taps (legacy or row-pair cache layout)
  auto wrow_of = [&](int a) -> const float* {
    if constexpr (PW) return a < (wn & ~1) ? rw.wc + (a >> 1) * wn * NT * 2 + (a & 1) : rw.wl;
    else return rw.wc + (G == 2 ? (a >> 1) : a) * wn * NT;
  };
  auto wst_of = [&](int a) { return (PW && a < (wn & ~1)) ? 2 * NT : NT; };
  auto weight = [&](const float* wrow, int wst, int b, int dx, int dy, float ik) {
    if constexpr (CW) {
      return wrow[b * wst];
    } else {
      const float d = rs.ic - ik;
      return m_exp(-(float)(dx * dx + dy * dy) * P.inv2s - d * d * P.inv2c);
    }
  };
  if (all_front) {
#pragma unroll 1
    for (int a = (G == 2 ? rw.g : 0); a < wn; a += G) {
      const int dy = -wr + a * ws;
      const int pa = G == 2 ? 0 : (a & 1);
      const float sy = fy + (float)dy;
      const float rx = fmaf(H[1], sy, H[2]);
      const float ry = fmaf(H[4], sy, H[5]);
      const float rz = fmaf(H[7], sy, H[8]);
      const float* trow = rw.t + dy * rw.tw;
      const float* wrow = wrow_of(a);
      const int wst = wst_of(a);
      auto tap = [&](int b) {
        const int dx = -wr + b * ws;
        const float sx = fx + (float)dx;
        const float ik = tile_at(rw, trow + dx);
        const float w = weight(wrow, wst, b, dx, dy, ik);
        const float izz = m_rcp(fmaf(H[6], sx, rz));
        accumulate(pa, w, sample(fmaf(H[0], sx, rx) * izz, fmaf(H[3], sx, ry) * izz), ik);
      };
      if constexpr (WR != 0) {
#pragma unroll
        for (int b = 0; b < (2 * WR) / WS + 1; ++b) tap(b);
      } else {
#pragma unroll 1
        for (int b = 0; b < wn; ++b) tap(b);
      }
    }
  } else {
#pragma unroll 1
    for (int a = (G == 2 ? rw.g : 0); a < wn; a += G) {
      const int dy = -wr + a * ws;
      const int pa = G == 2 ? 0 : (a & 1);
      const float sy = fy + (float)dy;
      const float rx = fmaf(H[1], sy, H[2]);
      const float ry = fmaf(H[4], sy, H[5]);
      const float rz = fmaf(H[7], sy, H[8]);
      const float* trow = rw.t + dy * rw.tw;
      const float* wrow = wrow_of(a);
      const int wst = wst_of(a);
#pragma unroll 1
      for (int b = 0; b < wn; ++b) {
        const int dx = -wr + b * ws;
        const float sx = fx + (float)dx;
        const float ik = tile_at(rw, trow + dx);
        const float w = weight(wrow, wst, b, dx, dy, ik);
        // the reciprocal is replaced by 0 behind the camera so the discarded fetch coordinates stay finite
        const float zz = fmaf(H[6], sx, rz);
        const bool front = zz > 1e-8f;
        const float izz = front ? m_rcp(zz) : 0.0f;
        const float sv = sample(fmaf(H[0], sx, rx) * izz, fmaf(H[3], sx, ry) * izz);
        accumulate(pa, w, front ? sv : 0.0f, ik);
      }
    }
  }
  return ncc_finish(rs, pair_total<G>(rw, Ss), pair_total<G>(rw, SSs), pair_total<G>(rw, IS));
}

template <int WR, int WS, bool CW, int NT, bool TEX = false, int G = 1>
__device__ __forceinline__ float ncc_cost(const PsRun& P, const RefWin& rw, const RefStats& rs, const PsLevel& S,
                                          const float* H, int x, int y, int& nwin) {
  if (!ncc_begin(rs, S, H, (float)x, (float)y)) return 2.0f;
  nwin++;
  return ncc_window<WR, WS, CW, NT, TEX, G>(P, rw, rs, S, H, x, y);
}

// ================================================================================ row-pair tap loops (f32x2)
// The window sums with rows 2p (even) and 2p+1 (odd) in the two halves of f32x2 pairs.  The even-row and odd-row
// partial sums of the parity contract advance in exactly the order of ncc_window, so the bits are the same, and each
// pair operation takes one issue slot for two taps.  Sources are sampled by plane loads, a texture gather, or the
// warp's staged source box (shared memory).
enum { SMP_LOAD = 0, SMP_TEX = 1, SMP_BOX = 2 };

// The warp's staged box: box[r·PS_BOX_P + c] holds texel (gx0 + c, gy0 + r) of the source (0 outside the image);
// mx = 1.5·2^23 - gx0 and my = 1.5·2^23 - gy0; the taps address it with 32-bit shared-memory addresses.
struct BoxRef {
  unsigned sbase;  // shared address of the box minus 4·(P + 1)·bits(1.5·2^23), mod 2^32
  float mx, my;
#if PS_CHECKED
  unsigned box;  // shared address of the box
  unsigned long long* fault;
#endif
};
// A BoxRef for the samplers that do not read a box (plane loads, texture).
__device__ __forceinline__ BoxRef no_box(const PsRun& P) {
  BoxRef b{0u, 0.f, 0.f};
#if PS_CHECKED
  b.box = 0u;
  b.fault = P.fault;
#endif
  return b;
}
// Checked build: the box texel q (byte address) and its 2 × 2 footprint inside the box.
__device__ __forceinline__ bool box_in(const BoxRef& bx, unsigned q) {
#if PS_CHECKED
  return PS_IN(bx.fault, PS_SITE_BOX, (long long)((q - bx.box) >> 2), 0, PS_BOX_P * PS_BOX_H - PS_BOX_P - 1);
#else
  return true;
#endif
}

// Reciprocal of a pair given nz = -z: m_rcp lane by lane (rcp.approx, then the FMA correction as pair operations).
__device__ __forceinline__ float2 m_rcp2(float2 nz) {
  float2 r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(-nz.x));
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(-nz.y));
#if PS_FAST
  return r;
#else
  return v_fma(r, v_fma(nz, r, v_splat(1.0f)), r);
#endif
}

// Bilinear samples of a pair of taps: the arithmetic of src_sample lane by lane, with the footprint from the plane,
// the texture or the box.  Box addressing: F = (u + mx) rounded toward -inf is floor(u) - gx0 + 1.5·2^23 exactly (u
// lies within the box, |gx0| < 2^15), so floor(u) = F - mx exactly and the bits of F are bits(1.5·2^23) + the box
// column; the box offset is therefore bits(Fv)·P + bits(Fu) - (P + 1)·bits(1.5·2^23), taken mod 2^32.
constexpr unsigned kBoxBias = 0u - 4u * (unsigned)(PS_BOX_P + 1) * 0x4B400000u;

__device__ __forceinline__ float lds(unsigned a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}
template <int OFF>
__device__ __forceinline__ float lds_off(unsigned a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1+%2];" : "=f"(v) : "r"(a), "n"(OFF));
  return v;
}

template <int SMP>
__device__ __forceinline__ float2 sample_pair(const PsLevel& S, const BoxRef& bx, float2 u, float2 v) {
  if constexpr (SMP == SMP_BOX) {
    const float2 mx = v_splat(bx.mx), my = v_splat(bx.my);
    const float2 fu = v_add_rm(u, mx), fv = v_add_rm(v, my);
    const float2 ax = v_sub(u, v_sub(fu, mx));
    const float2 ay = v_sub(v, v_sub(fv, my));
    // byte address = base + 4·(bits(Fv)·P + bits(Fu)) with the constant part folded into bx.sbase
    const unsigned qa = (unsigned)__float_as_int(fv.x) * (4u * PS_BOX_P) + bx.sbase + 4u * (unsigned)__float_as_int(fu.x);
    const unsigned qb = (unsigned)__float_as_int(fv.y) * (4u * PS_BOX_P) + bx.sbase + 4u * (unsigned)__float_as_int(fu.y);
#if PS_CHECKED
    if (!box_in(bx, qa) || !box_in(bx, qb)) return make_float2(0.f, 0.f);
#endif
    const float2 p00 = make_float2(lds(qa), lds(qb));
    const float2 p10 = make_float2(lds_off<4>(qa), lds_off<4>(qb));
    const float2 p01 = make_float2(lds_off<4 * PS_BOX_P>(qa), lds_off<4 * PS_BOX_P>(qb));
    const float2 p11 = make_float2(lds_off<4 * PS_BOX_P + 4>(qa), lds_off<4 * PS_BOX_P + 4>(qb));
    const float2 top = v_fma(ax, v_sub(p10, p00), p00);
    const float2 bot = v_fma(ax, v_sub(p11, p01), p01);
    return v_fma(ay, v_sub(bot, top), top);
  } else if constexpr (SMP == SMP_TEX) {
    // scalar per lane: the gather's four texels feed the bilinear directly (no repacking into pairs); floorf, not the
    // FMA-pipe add.rm floor of the box path, which measured 5 % slower here (more registers in the unrolled loop)
    return make_float2(src_sample_tex(S.tex, u.x, v.x), src_sample_tex(S.tex, u.y, v.y));
  } else {
#if PS_CHECKED
    unsigned long long* const fault = bx.fault;
#else
    unsigned long long* const fault = nullptr;
#endif
    return make_float2(src_sample(S.img, S.pitch, (float)S.w, (float)S.h, u.x, v.x, fault),
                       src_sample(S.img, S.pitch, (float)S.w, (float)S.h, u.y, v.y, fault));
  }
}

template <int SMP>
__device__ __forceinline__ float sample_one(const PsLevel& S, const BoxRef& bx, float u, float v) {
  if constexpr (SMP == SMP_BOX) {
    const float fu = __fadd_rd(u, bx.mx), fv = __fadd_rd(v, bx.my);
    const float ax = u - (fu - bx.mx), ay = v - (fv - bx.my);
    const unsigned q = (unsigned)__float_as_int(fv) * (4u * PS_BOX_P) + bx.sbase + 4u * (unsigned)__float_as_int(fu);
#if PS_CHECKED
    if (!box_in(bx, q)) return 0.f;
#endif
    const float p00 = lds(q), p10 = lds_off<4>(q), p01 = lds_off<4 * PS_BOX_P>(q), p11 = lds_off<4 * PS_BOX_P + 4>(q);
    const float top = fmaf(ax, p10 - p00, p00);
    const float bot = fmaf(ax, p11 - p01, p01);
    return fmaf(ay, bot - top, top);
  } else if constexpr (SMP == SMP_TEX) {
    return src_sample_tex(S.tex, u, v);
  } else {
#if PS_CHECKED
    return src_sample(S.img, S.pitch, (float)S.w, (float)S.h, u, v, bx.fault);
#else
    return src_sample(S.img, S.pitch, (float)S.w, (float)S.h, u, v);
#endif
  }
}

// Window sums of a window whose four corner taps lie in front of the source camera (every tap then does), with the
// row-pair weight cache.  Rows 2p / 2p+1 go through the pair loop; the last row of an odd window is scalar and adds
// into the even-row sums, as in ncc_window.  UNROLL unrolls the pair loop over the window columns (the staged path);
// the rolled form keeps the fallback's code small (instruction-cache footprint of the staged kernel).
template <int WR, int WS, int NT, int SMP, bool UNROLL>
__device__ __forceinline__ float ncc_window_pairs(const RefWin& rw, const RefStats& rs, const PsLevel& S, const float* H,
                                                  int x, int y, const BoxRef& bx) {
  constexpr int wr = WR, ws = WS, wn = (2 * WR) / WS + 1, np = wn / 2;
  const float fx = (float)x, fy = (float)y;
  float2 Ss = v_splat(0.f), SSs = v_splat(0.f), IS = v_splat(0.f);
  const float2 h0 = v_splat(H[0]), h1 = v_splat(H[1]), h2 = v_splat(H[2]), h3 = v_splat(H[3]), h4 = v_splat(H[4]),
               h5 = v_splat(H[5]), nh6 = v_splat(-H[6]), nh7 = v_splat(-H[7]), nh8 = v_splat(-H[8]);
#pragma unroll 1
  for (int p = 0; p < np; ++p) {
    const int dy = -wr + 2 * p * ws;
    const float2 sy = make_float2(fy + (float)dy, fy + (float)(dy + ws));
    const float2 rx = v_fma(h1, sy, h2), ry = v_fma(h4, sy, h5), nrz = v_fma(nh7, sy, nh8);
    const float* t0 = rw.t + dy * rw.tw;
    const float* t1 = t0 + ws * rw.tw;
    const float* wp = rw.wc + p * wn * NT * 2;
    auto tap = [&](int dx, float sxf, const float* wq) {
      const float2 sx = v_splat(sxf);
      const float2 ik = make_float2(tile_at(rw, t0 + dx), tile_at(rw, t1 + dx));
      const float2 w = *reinterpret_cast<const float2*>(wq);
      const float2 izz = m_rcp2(v_fma(nh6, sx, nrz));
      const float2 sv = sample_pair<SMP>(S, bx, v_mul(v_fma(h0, sx, rx), izz), v_mul(v_fma(h3, sx, ry), izz));
      const float2 wsv = v_mul(w, sv);
      Ss = v_add(Ss, wsv);
      SSs = v_fma(wsv, sv, SSs);
      IS = v_fma(wsv, ik, IS);
    };
    if constexpr (UNROLL) {
#pragma unroll
      for (int b = 0; b < wn; ++b) tap(-wr + b * ws, fx + (float)(-wr + b * ws), wp + b * NT * 2);
    } else {
      int dx = -wr;
      float sxf = fx + (float)(-wr);
      const float* wq = wp;
#pragma unroll 1
      for (int b = 0; b < wn; ++b) {
        tap(dx, sxf, wq);
        dx += ws;
        sxf += (float)ws;
        wq += NT * 2;
      }
    }
  }
  if constexpr ((wn & 1) != 0) {
    const int dy = -wr + (wn - 1) * ws;
    const float sy = fy + (float)dy;
    const float rx = fmaf(H[1], sy, H[2]), ry = fmaf(H[4], sy, H[5]), rz = fmaf(H[7], sy, H[8]);
    const float* t0 = rw.t + dy * rw.tw;
    auto tap = [&](int b, int dx, float sx) {
      const float ik = tile_at(rw, t0 + dx);
      const float w = rw.wl[b * NT];
      const float izz = m_rcp(fmaf(H[6], sx, rz));
      const float sv = sample_one<SMP>(S, bx, fmaf(H[0], sx, rx) * izz, fmaf(H[3], sx, ry) * izz);
      const float wsv = w * sv;
      Ss.x = Ss.x + wsv;
      SSs.x = fmaf(wsv, sv, SSs.x);
      IS.x = fmaf(wsv, ik, IS.x);
    };
    if constexpr (UNROLL) {
#pragma unroll
      for (int b = 0; b < wn; ++b) tap(b, -wr + b * ws, fx + (float)(-wr + b * ws));
    } else {
      int dx = -wr;
      float sx = fx + (float)(-wr);
#pragma unroll 1
      for (int b = 0; b < wn; ++b) {
        tap(b, dx, sx);
        dx += ws;
        sx += (float)ws;
      }
    }
  }
  return ncc_finish(rs, Ss.x + Ss.y, SSs.x + SSs.y, IS.x + IS.y);
}

// Corner test of ncc_window: the four corner taps in front of the source camera.
template <int WR>
__device__ __forceinline__ bool window_front(const float* H, float fx, float fy) {
  const float sx0 = fx + (float)(-WR), sx1 = fx + (float)WR;
  const float rz0 = fmaf(H[7], fy + (float)(-WR), H[8]), rz1 = fmaf(H[7], fy + (float)WR, H[8]);
  return fmaf(H[6], sx0, rz0) > 1e-8f && fmaf(H[6], sx1, rz0) > 1e-8f && fmaf(H[6], sx0, rz1) > 1e-8f &&
         fmaf(H[6], sx1, rz1) > 1e-8f;
}

// One lane's window with the row-pair loops (the prologue must have passed): pair loop when the window is wholly in
// front, otherwise the guarded loop of ncc_window on the row-pair cache.
template <int WR, int WS, int NT, bool TEX>
__device__ __forceinline__ float ncc_window_lane(const PsRun& P, const RefWin& rw, const RefStats& rs,
                                                 const PsLevel& S, const float* H, int x, int y) {
  constexpr int smp = TEX ? SMP_TEX : SMP_LOAD;
  if (window_front<WR>(H, (float)x, (float)y))
    return ncc_window_pairs<WR, WS, NT, smp, true>(rw, rs, S, H, x, y, no_box(P));
  return ncc_window<WR, WS, true, NT, TEX, 1, true>(P, rw, rs, S, H, x, y);
}

// ------------------------------------------------------------------------------------------- TMA staging
// Tensor maps (built by the runtime for PS_TUNE_TMA) describe each bordered image plane as a 2-D f32 tensor of
// pitch × (h + 2·PS_BORDER) elements whose origin is the plane's allocation (texel (-PS_BORDER, -PS_BORDER)), so a
// texel (X, Y) is element (X + PS_BORDER, Y + PS_BORDER); elements outside the tensor read 0, like the border.  Per
// (view, level) the table holds two maps: the reference tile box (PsRun.tma_tile_w × PS_HALF_PH + 2·wr) and the
// source box (PS_BOX_P × PS_BOX_H).  Loads are plain 2-D tiled loads into this CTA's shared memory (no multicast),
// completed on an mbarrier with a byte count.
__device__ __forceinline__ const void* tmap(const PsRun& P, int view, int which) {
  return (const unsigned char*)P.tmaps + ((size_t)(view * P.nlevels + P.level) * 2 + which) * 128;
}
__device__ __forceinline__ void mbar_init(unsigned bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
// One thread: expect `bytes` on the barrier and start the 2-D load of the box at element (x, y) (x·4 must be a
// multiple of 16) into shared memory at dst (128-byte aligned).
__device__ __forceinline__ void tma_load_2d(unsigned dst, const void* map, int x, int y, unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
// Bounded wait for the barrier's phase `parity` to complete.  After PS_TMA_SPIN_LIMIT polls the error word (when
// set) is marked, the wait is repeated once more with the same bound (the copy may still land), and false returns;
// the caller's data is then unreliable and the run reports PS_ETIMEOUT.
#define PS_TMA_SPIN_LIMIT (1u << 20)
__device__ __forceinline__ bool mbar_wait(const PsRun& P, unsigned bar, unsigned parity) {
  for (int round = 0; round < 2; ++round) {
    for (unsigned i = 0; i < PS_TMA_SPIN_LIMIT; ++i) {
      unsigned done;
      asm volatile(
          "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(done)
          : "r"(bar), "r"(parity)
          : "memory");
      if (done) return round == 0;
    }
    if (round == 0 && P.queue) atomicCAS(P.queue + 1, 0u, 2u);
  }
  return false;
}
// Shared-memory reads of a buffer made by the generic proxy are ordered before a following TMA write into it.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// What the warp's box holds: texels [ox, ox + PS_BOX_P) × [oy, oy + PS_BOX_H) of the plane at src (warp-uniform).
struct BoxState {
  const float* src;
  int ox, oy;
  unsigned bar, phase;  // TMA staging: the warp's mbarrier (shared address) and its next phase parity
  // profiling: this lane's windows read from the box, restages (counted on every lane), and this lane's windows left
  // to the per-lane loops because the footprint bound failed, the warp's request was too wide or too tall, or too few
  // lanes were active
  int nstaged, nrestage, nbound, nwide, ntall, nfew;
};

// Warp-collective NCC cost (every lane of the warp calls it; `act` marks the lanes that want this window).
//
// The lanes' windows usually overlap in the source (neighbouring pixels, similar planes), so the warp stages the
// union of their footprints into its shared-memory box once and every tap reads its 2×2 texels from there instead of
// the texture unit.  Footprint bound: the tap position is a projective function of the tap with a positive
// denominator over the window, so its exact value lies between the values at the four corner taps.  The computed
// positions differ from the exact ones by at most 2^-23·(Tu + |u|·Tz)/zmin + 2^-23·|u| (Tu, Tz the sums of the
// magnitudes of the homography terms at the window's extreme coordinates); with Tu, Tv, (|u|+|v|+1)·Tz ≤ 2^14·zmin
// and |u|, |v| < 2^14 that is below 2^-7, so the texels [floor(umin - 1/64), floor(umax + 1/64) + 1] of the computed
// corner positions cover every texel a tap reads.  The box is reused while the requested footprints fit inside it;
// a restage centres the box on the request and copies it with 16-byte cp.async chunks.  Windows that fail the bound,
// a request wider than PS_BOX_P - 3 or taller than PS_BOX_H texels, or fewer than PS_STAGE_MIN_LANES active lanes use
// the per-lane loops.  All paths give the same bits.
template <int WR, int WS, int NT, bool TEX, bool TMA>
__device__ __forceinline__ float ncc_cost_warp(const PsRun& P, const RefWin& rw, const RefStats& rs, const PsLevel& S,
                                               int src, const float* H, int x, int y, bool act, int& nwin, float* box,
                                               BoxState& bs) {
  const float fx = (float)x, fy = (float)y;
  act = act && ncc_begin(rs, S, H, fx, fy);
  const unsigned am = __ballot_sync(0xffffffffu, act);
  if (am == 0u) return 2.0f;
  if (act) nwin++;
  bool front = false, fits = false;
  int lx = 0x7fffffff, ly = 0x7fffffff, hx = -0x7fffffff, hy = -0x7fffffff;
  if (act) {
    const float sx0 = fx + (float)(-WR), sx1 = fx + (float)WR, sy0 = fy + (float)(-WR), sy1 = fy + (float)WR;
    const float rz0 = fmaf(H[7], sy0, H[8]), rz1 = fmaf(H[7], sy1, H[8]);
    const float z00 = fmaf(H[6], sx0, rz0), z10 = fmaf(H[6], sx1, rz0);
    const float z01 = fmaf(H[6], sx0, rz1), z11 = fmaf(H[6], sx1, rz1);
    front = z00 > 1e-8f && z10 > 1e-8f && z01 > 1e-8f && z11 > 1e-8f;
    if (front) {
      const float rx0 = fmaf(H[1], sy0, H[2]), rx1 = fmaf(H[1], sy1, H[2]);
      const float ry0 = fmaf(H[4], sy0, H[5]), ry1 = fmaf(H[4], sy1, H[5]);
      const float i00 = m_rcp(z00), i10 = m_rcp(z10), i01 = m_rcp(z01), i11 = m_rcp(z11);
      const float u00 = fmaf(H[0], sx0, rx0) * i00, u10 = fmaf(H[0], sx1, rx0) * i10;
      const float u01 = fmaf(H[0], sx0, rx1) * i01, u11 = fmaf(H[0], sx1, rx1) * i11;
      const float v00 = fmaf(H[3], sx0, ry0) * i00, v10 = fmaf(H[3], sx1, ry0) * i10;
      const float v01 = fmaf(H[3], sx0, ry1) * i01, v11 = fmaf(H[3], sx1, ry1) * i11;
      const float umin = fminf(fminf(u00, u10), fminf(u01, u11)), umax = fmaxf(fmaxf(u00, u10), fmaxf(u01, u11));
      const float vmin = fminf(fminf(v00, v10), fminf(v01, v11)), vmax = fmaxf(fmaxf(v00, v10), fmaxf(v01, v11));
      const float zmin = fminf(fminf(z00, z10), fminf(z01, z11));
      const float mx = fmaxf(fabsf(sx0), fabsf(sx1)), my = fmaxf(fabsf(sy0), fabsf(sy1));
      const float tu = fabsf(H[0]) * mx + fabsf(H[1]) * my + fabsf(H[2]);
      const float tv = fabsf(H[3]) * mx + fabsf(H[4]) * my + fabsf(H[5]);
      const float tz = fabsf(H[6]) * mx + fabsf(H[7]) * my + fabsf(H[8]);
      const float ua = fmaxf(fabsf(umin), fabsf(umax)), va = fmaxf(fabsf(vmin), fabsf(vmax));
      const float lim = 16384.0f * zmin;
      fits = zmin < 1e30f && tu <= lim && tv <= lim && (ua + va + 1.0f) * tz <= lim && ua < 16384.0f && va < 16384.0f;
      if (fits) {
        lx = (int)floorf(umin - 0.015625f);
        hx = (int)floorf(umax + 0.015625f) + 1;
        ly = (int)floorf(vmin - 0.015625f);
        hy = (int)floorf(vmax + 0.015625f) + 1;
      }
    }
  }
  const bool allfit = __all_sync(0xffffffffu, !act || fits);
  const bool many = __popc(am) >= PS_STAGE_MIN_LANES;
  if (P.stage_count && act) {
    bs.nbound += !allfit;
    bs.nfew += allfit && !many;
  }
  if (allfit && many) {
    const int gx0 = __reduce_min_sync(0xffffffffu, lx), gx1 = __reduce_max_sync(0xffffffffu, hx);
    const int gy0 = __reduce_min_sync(0xffffffffu, ly), gy1 = __reduce_max_sync(0xffffffffu, hy);
    const bool narrow = gx1 - gx0 + 1 <= PS_BOX_P - 3, low = gy1 - gy0 + 1 <= PS_BOX_H;
    if (P.stage_count && act) {
      bs.nwide += !narrow;
      bs.ntall += narrow && !low;
    }
    if (narrow && low) {
      if (!(S.img == bs.src && gx0 >= bs.ox && gx1 < bs.ox + PS_BOX_P && gy0 >= bs.oy && gy1 < bs.oy + PS_BOX_H)) {
        // Restage, centred on the request: origin x ≡ 2 (mod 4), so every 16-byte chunk of a plane row is aligned
        // (rows start 2 floats after a 128-byte boundary); chunks outside the plane's allocated rows are zero-filled,
        // inside they read the image or its zero border and padding.
        const int xlo = gx1 - (PS_BOX_P - 1), ylo = gy1 - (PS_BOX_H - 1);
        int ox = (xlo + gx0) >> 1;
        ox -= (ox - 2) & 3;
        if (ox < xlo) ox += 4;
        const int oy = (ylo + gy0) >> 1;
        __syncwarp();  // every lane is done with the previous box
        const int lane = threadIdx.x & 31;
        const unsigned sbase = (unsigned)__cvta_generic_to_shared(box);
        if constexpr (TMA) {
          // one 2-D tensor load of the whole box (x = ox + PS_BORDER ≡ 0 mod 4: 16-byte aligned); outside the
          // plane's tensor the box reads 0, as the cp.async path's zero-filled chunks do
          if (lane == 0) {
            fence_proxy_async();
            tma_load_2d(sbase, tmap(P, src, 1), ox + PS_BORDER, oy + PS_BORDER, bs.bar, PS_BOX_P * PS_BOX_H * 4u);
          }
          mbar_wait(P, bs.bar, bs.phase);
          bs.phase ^= 1u;
        } else {
#pragma unroll 2
          for (int i = lane; i < PS_BOX_H * (PS_BOX_P / 4); i += 32) {
            const int r = i / (PS_BOX_P / 4), q = i - r * (PS_BOX_P / 4);
            const int X = ox + 4 * q, Y = oy + r;
            const bool in = Y >= -PS_BORDER && Y < S.h + PS_BORDER && X >= -PS_BORDER && X + 4 <= S.pitch - PS_BORDER;
            const float* srcp = in ? S.img + (long long)Y * S.pitch + X : S.img - PS_BORDER;  // aligned; 0 bytes read
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sbase + 4u * (unsigned)(r * PS_BOX_P + 4 * q)),
                         "l"(srcp), "r"(in ? 16 : 0)
                         : "memory");
          }
          asm volatile("cp.async.wait_all;\n" ::: "memory");
        }
        __syncwarp();
        bs.src = S.img;
        bs.ox = ox;
        bs.oy = oy;
        bs.nrestage++;
      }
      if (act) bs.nstaged++;
      BoxRef bx{(unsigned)__cvta_generic_to_shared(box) + kBoxBias, 12582912.0f - (float)bs.ox, 12582912.0f - (float)bs.oy};
#if PS_CHECKED
      bx.box = (unsigned)__cvta_generic_to_shared(box);
      bx.fault = P.fault;
#endif
      return act ? ncc_window_pairs<WR, WS, NT, SMP_BOX, true>(rw, rs, S, H, x, y, bx) : 2.0f;
    }
  }
  if (!act) return 2.0f;
  if (front)
    return ncc_window_pairs<WR, WS, NT, TEX ? SMP_TEX : SMP_LOAD, true>(rw, rs, S, H, x, y, no_box(P));
  return ncc_window<WR, WS, true, NT, TEX, 1, true>(P, rw, rs, S, H, x, y);
}

// Forward/backward reprojection error through the source snapshot (patchmatch.cu:292-314); INF on failure.
#define PS_INF_ERR 1e30f
__device__ float geo_error(const PsRun& P, const PsLevel& R, const PsLevel& S, const PsPair& pr, int x, int y,
                           float d) {
  long long off = P.snap_off[pr.src];
  if (off < 0) return PS_INF_ERR;
  float3 X = make_float3(((float)x - R.cx) / R.fx * d, ((float)y - R.cy) / R.fy * d, d);
  float xj = pr.r[0] * X.x + pr.r[1] * X.y + pr.r[2] * X.z + pr.t[0];
  float yj = pr.r[3] * X.x + pr.r[4] * X.y + pr.r[5] * X.z + pr.t[1];
  float zj = pr.r[6] * X.x + pr.r[7] * X.y + pr.r[8] * X.z + pr.t[2];
  if (!(zj > 1e-8f)) return PS_INF_ERR;
  float u = S.fx * xj / zj + S.cx, v = S.fy * yj / zj + S.cy;
  float uf = floorf(u + 0.5f), vf = floorf(v + 0.5f);
  if (!(uf >= 0.f && vf >= 0.f && uf < (float)S.w && vf < (float)S.h)) return PS_INF_ERR;
  if (!PS_IN(P.fault, PS_SITE_SNAPSHOT, off + (long long)vf * S.w + (long long)uf, 0, P.snap_pixels)) return PS_INF_ERR;
  float dj = __ldg(P.snap + off + (long long)vf * S.w + (long long)uf);
  if (!(dj > 0.f)) return PS_INF_ERR;
  float3 Yj = make_float3((u - S.cx) / S.fx * dj, (v - S.cy) / S.fy * dj, dj);
  float3 q = make_float3(Yj.x - pr.t[0], Yj.y - pr.t[1], Yj.z - pr.t[2]);
  float Yx = pr.r[0] * q.x + pr.r[3] * q.y + pr.r[6] * q.z;
  float Yy = pr.r[1] * q.x + pr.r[4] * q.y + pr.r[7] * q.z;
  float Yz = pr.r[2] * q.x + pr.r[5] * q.y + pr.r[8] * q.z;
  if (!(Yz > 1e-8f)) return PS_INF_ERR;
  float cx = R.fx * Yx / Yz + R.cx - (float)x, cy = R.fy * Yy / Yz + R.cy - (float)y;
  return sqrtf(cx * cx + cy * cy);
}

// (photometric cost, truncated geometric error) of one hypothesis × one source (patchmatch.cu:316-324).
template <int WR, int WS, bool CW, int NT, bool TEX = false, int G = 1>
__device__ __forceinline__ float pair_cost(const PsRun& P, const RefWin& rw, const RefStats& rs, const PsLevel& R,
                                           const PsLevel& S, const PsPair& pr, const PsLPair& lp, int x, int y,
                                           float4 h, float* geo, int& nwin) {
  float H[9];
  float c = 2.0f;
  if (homography(R, lp, (float)x, (float)y, h, H)) c = ncc_cost<WR, WS, CW, NT, TEX, G>(P, rw, rs, S, H, x, y, nwin);
  if (P.geometric) *geo = fminf(geo_error(P, R, S, pr, x, y, h.w), P.gmax);
  return c;
}

// Random normal toward the camera (patchmatch.cu:348-361), random depth (:363-366), perturbed normal (:368-384).
__device__ float3 random_normal(u64& st, float3 ray) {
  float3 n = make_float3(0.f, 0.f, -1.f);
  for (int k = 0; k < 64; ++k) {
    float v1 = 2.f * rnd(st) - 1.f, v2 = 2.f * rnd(st) - 1.f;
    float s = v1 * v1 + v2 * v2;
    if (s < 1.f && s > 0.f) {
      float r = 2.f * sqrtf(1.f - s);
      n = make_float3(v1 * r, v2 * r, 1.f - 2.f * s);
      break;
    }
  }
  if (dot3(n, ray) > 0.f) n = make_float3(-n.x, -n.y, -n.z);
  return n;
}
__device__ __forceinline__ float random_depth(u64& st, float dmin, float dmax) {
  float a = 1.f / dmax, b = 1.f / dmin;
  return 1.f / (a + rnd(st) * (b - a));
}
__device__ float3 perturb_normal(u64& st, float3 n, float3 ray, float phi) {
  float3 a = random_normal(st, make_float3(0.f, 0.f, 0.f));
  float3 ax = cross3(a, n);
  float l2 = dot3(ax, ax);
  float ang = rnd(st) * phi;
  if (l2 < 1e-12f) return n;
  ax = nrm3(ax);
  float3 bn = cross3(ax, n);
  for (int k = 0; k < 4; ++k) {
    float sa, ca;
    m_sincos(ang, &sa, &ca);
    float3 m = make_float3(n.x * ca + bn.x * sa, n.y * ca + bn.y * sa, n.z * ca + bn.z * sa);
    if (dot3(m, ray) < 0.f) return nrm3(m);
    ang *= 0.5f;
  }
  return n;
}

// Triangulation × incidence × resolution prior (patchmatch.cu:388-422).
__device__ float view_prior(const PsRun& P, const PsLevel& R, const PsPair& pr, const float* H, bool hok, int x, int y,
                            float4 h, int wr) {
  if (!hok) return 0.f;
  float3 ray = pixel_ray(R, x, y);
  float3 X = make_float3(ray.x * h.w, ray.y * h.w, h.w);
  float3 S = make_float3(pr.c[0] - X.x, pr.c[1] - X.y, pr.c[2] - X.z);
  float ls = sqrtf(dot3(S, S)), lx = sqrtf(dot3(X, X));
  if (ls <= 0.f || lx <= 0.f) return 0.f;
  float cost = -dot3(S, X) / (ls * lx);
  float tri = 1.f;
  if (cost > P.cos_tri_min) {
    float s = 1.f - (1.f - cost) / (1.f - P.cos_tri_min);
    tri = fminf(fmaxf(1.f - s * s, 0.f), 1.f);
  }
  float cphi = dot3(S, make_float3(h.x, h.y, h.z)) / ls;
  float xi = 1.f - fmaxf(0.f, cphi);
  float inc = m_exp(-xi * xi * P.inv2inc);
  float r = (float)wr;
  float cxs[4] = {x - r, x - r, x + r, x + r};
  float cys[4] = {y - r, y + r, y + r, y - r};
  float px[4], py[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float z = H[6] * cxs[k] + H[7] * cys[k] + H[8];
    if (!(z > 1e-8f)) return 0.f;
    px[k] = (H[0] * cxs[k] + H[1] * cys[k] + H[2]) / z;
    py[k] = (H[3] * cxs[k] + H[4] * cys[k] + H[5]) / z;
  }
  float area = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) area += px[k] * py[(k + 1) & 3] - px[(k + 1) & 3] * py[k];
  area = 0.5f * fabsf(area);
  float aref = (2.f * r + 1.f) * (2.f * r + 1.f);
  if (!(area > 0.f)) return 0.f;
  float res = fminf(area / aref, aref / area);
  return tri * inc * res;
}

// Propagation offsets of the 8 regions in order (patchmatch.cu:424-436, :480-490): regions 0-3 are the V shapes
// (0,-1),(±1,-2),(±2,-3),(±3,-4) rotated up→right→down→left by (dx,dy)→(-dy,dx); regions 4-7 the bands
// (0,-3),(0,-5),…,(0,-23) with the same rotations.  Every offset has odd |dx|+|dy| (opposite colour).
__constant__ int2 c_prop[72];

__device__ __forceinline__ int find_item(const PsRun& P, int cta) {
  int lo = 0, hi = P.nitems - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (P.items[mid].tile0 <= cta) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Checked build: the item's view, its pixels in the state arrays, its source count and source views; the self-test
// probe (PsRun.probe) tests one index past the end of the state arrays here, so no access follows it.  CTA-uniform,
// so a kernel may return on false before its first barrier.  Always true in the other builds.
__device__ __forceinline__ bool item_ok(const PsRun& P, const PsItem& it) {
#if PS_CHECKED
  if (P.probe && blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0)
    (void)PS_IN(P.fault, PS_SITE_PROBE, P.state_pixels, 0, P.state_pixels);
  if (!PS_IN(P.fault, PS_SITE_SOURCE, it.view, 0, P.nviews_all)) return false;
  if (!PS_IN(P.fault, PS_SITE_STATE, it.off, 0, P.state_pixels) ||
      !PS_IN(P.fault, PS_SITE_STATE, it.off + (long long)it.w * it.h - 1, 0, P.state_pixels))
    return false;
  const int nsrc = P.views[it.view].nsrc;
  if (!PS_IN(P.fault, PS_SITE_SOURCE, nsrc, 0, PS_MAXSRC + 1)) return false;
  for (int j = 0; j < nsrc; ++j)
    if (!PS_IN(P.fault, PS_SITE_SOURCE, P.pairs[(size_t)it.view * PS_MAXSRC + j].src, 0, P.nviews_all)) return false;
#endif
  return true;
}

// ================================================================================ half step (patchmatch.cu:439-657)
// Warp-aggregated add of the per-thread NCC window count (threads that already returned do not take part).
__device__ __forceinline__ void count_windows(const PsRun& P, int nwin) {
  if (!P.ncc_count) return;
  const unsigned m = __activemask();
  const unsigned s = __reduce_add_sync(m, (unsigned)nwin);
  if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && s) atomicAdd(P.ncc_count, (unsigned long long)s);
}

// Profiling: refinement windows skipped because the candidate's partial cost had reached the best cost (the
// half-step kernels' early exit), into staged-statistics slot 6 of the launch's kind.
__device__ __forceinline__ void count_skipped(const PsRun& P, int n) {
  if (!P.stage_count) return;
  const unsigned m = __activemask();
  const unsigned s = __reduce_add_sync(m, (unsigned)n);
  if ((int)(threadIdx.x & 31) == __ffs(m) - 1 && s) atomicAdd(P.stage_count + 6, (unsigned long long)s);
}

// Half-step tile geometry for G lanes per pixel: G = 1 -> 32 × 8 pixels (a warp = 16 active columns × 2 rows);
// G = 2 -> 16 × 8 pixels (a warp = 8 active columns × 2 rows × 2 lanes).  The shared tile's row pitch is padded so
// that the lanes of one warp read 32 distinct banks: even for G = 1, ≡ 16 (mod 32) for G = 2.  The staged kernel's
// warp (4 active columns × 8 rows) needs a pitch ≡ 4 or 12 (mod 16): its same-parity rows then fall 8 banks apart
// and the checkerboard puts the other rows on the other bank parity.
__host__ __device__ constexpr int half_pw(int G) { return G == 2 ? PS_HALF2_PW : PS_HALF_PW; }
__host__ __device__ constexpr int half_tw(int G, int wr) {
  return G == 2 ? (((PS_HALF2_PW + 2 * wr) + 15) / 32) * 32 + 16 : PS_HALF_PW + 2 * wr;
}
__host__ __device__ constexpr int half_tw_staged(int wr) { return PS_HALF_ST_TW(wr); }

// ---------------------------------------------------------------------------- per-pixel PatchMatch logic
// Shared by the half-step kernels; each helper is the reference's step verbatim (patchmatch.cu line ranges cited).

// 1. Candidates: the current plane and the best-cost neighbour of each of the 8 regions, transferred onto this
// pixel's ray (patchmatch.cu:477-511).
__device__ __forceinline__ void propagation_candidates(const PsLevel& R, const float4* pl, const float* co, int x, int y,
                                                       int w, int h, float3 ray, float4* hyp) {
  hyp[0] = pl[y * w + x];
#pragma unroll 1
  for (int r = 0; r < 8; ++r) {
    const int k0 = r < 4 ? r * 7 : 28 + (r - 4) * 11;
    const int cnt = r < 4 ? 7 : 11;
    float best = 1e30f;
    int bq = -1, bx = 0, by = 0;
    for (int k = 0; k < cnt; ++k) {
      const int2 o = c_prop[k0 + k];
      const int qx = x + o.x, qy = y + o.y;
      if (qx < 0 || qy < 0 || qx >= w || qy >= h) continue;
      const float c = co[qy * w + qx];
      if (c < best) {
        best = c;
        bq = qy * w + qx;
        bx = qx;
        by = qy;
      }
    }
    hyp[1 + r] = hyp[0];
    if (bq >= 0) {
      const float4 q = pl[bq];
      const float3 n = make_float3(q.x, q.y, q.z);
      const float3 rq = pixel_ray(R, bx, by);
      const float den = dot3(n, ray);
      if (den < -1e-6f && q.w > 0.f) {
        const float d = q.w * dot3(n, rq) / den;
        if (d > 0.f && isfinite(d)) hyp[1 + r] = make_float4(n.x, n.y, n.z, d);
      }
    }
  }
}

// 2. View selection and aggregation (patchmatch.cu:513-594): per source, votes over the 8 propagated hypotheses,
// the view weight, and the weighted cost sums of the 9 hypotheses; then the aggregated argmin.
struct ViewAgg {
  float num[9], numf[9];
  float den, denf, wbest;
  int vbest;
};
__device__ __forceinline__ void agg_init(ViewAgg& a) {
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    a.num[i] = 0.f;
    a.numf[i] = 0.f;
  }
  a.den = 0.f;
  a.wbest = 0.f;
  a.denf = 0.f;
  a.vbest = 255;
}
// The values that change between the half steps of a run: iteration, colour and the iteration's constants
// (patchmatch.rs:752-799: tau_good, eps and phi follow the iteration).  A launch per half step takes them from its
// PsRun; the persistent kernel from the run's phase table.
struct HalfPhase {
  int t, color;
  float tau_good, eps, phi;
};
__device__ __forceinline__ HalfPhase launch_phase(const PsRun& P) {
  return HalfPhase{P.t, P.color, P.tau_good, P.eps, P.phi};
}

// Source j with prior > 0: m, gg = photometric costs and truncated geometric errors of the 9 hypotheses; writes the
// view weight (or -prior) to *wvj.
__device__ __forceinline__ void agg_source(const PsRun& P, float tau_good, ViewAgg& a, const float* m, const float* gg,
                                           float prior, int j, int vprev, float* wvj) {
  int good = 0, bad = 0;
  float conf = 0.f;
#pragma unroll
  for (int i = 1; i < 9; ++i) {
    if (m[i] < tau_good) {
      good++;
      conf += m_exp(-m[i] * m[i] * P.inv2beta2);
    }
    if (m[i] > P.tau_bad) bad++;
  }
  const bool adopt = good > P.n1 && bad < P.n2;
  const bool isprev = j == vprev;
  const float wp = adopt ? (isprev ? 2.f : 1.f) * conf / (float)good : (isprev ? P.prev_w : 0.f);
  const float w2 = wp * prior;
  *wvj = w2 > 0.f ? w2 : -prior;
#pragma unroll
  for (int i = 0; i < 9; ++i) a.numf[i] += prior * (m[i] + P.lambda * gg[i]);
  a.denf += prior;
  if (w2 > 0.f) {
#pragma unroll
    for (int i = 0; i < 9; ++i) a.num[i] += w2 * (m[i] + P.lambda * gg[i]);
    a.den += w2;
    if (w2 > a.wbest) {
      a.wbest = w2;
      a.vbest = j;
    }
  }
}
// Aggregated costs, the prior-weighted fallback (view weights become the priors, den = denf), the argmin (earliest on
// ties); returns the best hypothesis and its cost.
__device__ __forceinline__ void agg_finish(ViewAgg& a, const float4* hyp, int nsrc, float* wv, int wstride,
                                           float4& best, float& bcost) {
  float agg[9];
  int bi9 = 0;
  if (a.den > 0.f) {
#pragma unroll
    for (int i = 0; i < 9; ++i) agg[i] = a.num[i] / a.den;
  } else if (a.denf > 0.f) {
#pragma unroll
    for (int i = 0; i < 9; ++i) agg[i] = a.numf[i] / a.denf;
    for (int j = 0; j < nsrc; ++j) wv[j * wstride] = -wv[j * wstride];
    a.den = a.denf;
  } else {
#pragma unroll
    for (int i = 0; i < 9; ++i) agg[i] = 2.f;
  }
  float bagg = agg[0];
#pragma unroll
  for (int i = 1; i < 9; ++i)
    if (agg[i] < bagg) {
      bagg = agg[i];
      bi9 = i;
    }
  best = hyp[0];
#pragma unroll
  for (int i = 1; i < 9; ++i)
    if (i == bi9) best = hyp[i];
  bcost = bagg;
}

// 3. Refinement candidates (patchmatch.cu:596-628) and 4. the coarse-scale candidate (:629-653).  The draws come from
// the per-pixel RNG in the reference's order; a best plane with d <= 0 takes the random depth.
struct Refine {
  float3 n0, n_r, n_p;
  float d_r, d_p, bw;
  float4 qprior;
  int ncand;
};
// has_prior / qprior: the coarse-scale candidate (does not depend on the traversal).
__device__ __forceinline__ void refine_prior(const PsRun& P, long long g, float var, float3 ray, Refine& r) {
  bool has_prior = false;
  r.qprior = make_float4(0.f, 0.f, 0.f, 0.f);
  if (P.use_prior && var < P.weak_var) {
    r.qprior = P.prior[g];
    has_prior = r.qprior.w > 0.f && dot3(make_float3(r.qprior.x, r.qprior.y, r.qprior.z), ray) < 0.f;
  }
  r.ncand = has_prior ? 7 : 6;
}
__device__ __forceinline__ void refine_draw(const PsRun& P, const HalfPhase& ph, const PsView& vd, int pix, float3 ray,
                                            float4& best, Refine& r) {
  u64 st = rng_state(P.seed, vd.key, P.level, P.run_id, ph.t, ph.color, (u64)pix);
  r.d_r = random_depth(st, vd.dmin, vd.dmax);
  r.n_r = random_normal(st, ray);
  const float uu = 2.f * rnd(st) - 1.f;
  const float inv = best.w > 0.f ? (1.f / best.w) * (1.f + uu * ph.eps) : -1.f;
  r.d_p = inv > 0.f ? 1.f / inv : r.d_r;
  if (!(best.w > 0.f)) best.w = r.d_r;
  r.n0 = make_float3(best.x, best.y, best.z);
  r.n_p = perturb_normal(st, r.n0, ray, ph.phi);
  r.bw = best.w;
}
__device__ __forceinline__ float4 refine_candidate(const Refine& r, int c) {
  switch (c) {
    case 0: return make_float4(r.n0.x, r.n0.y, r.n0.z, r.d_r);
    case 1: return make_float4(r.n_r.x, r.n_r.y, r.n_r.z, r.bw);
    case 2: return make_float4(r.n_r.x, r.n_r.y, r.n_r.z, r.d_r);
    case 3: return make_float4(r.n0.x, r.n0.y, r.n0.z, r.d_p);
    case 4: return make_float4(r.n_p.x, r.n_p.y, r.n_p.z, r.bw);
    case 5: return make_float4(r.n_p.x, r.n_p.y, r.n_p.z, r.d_p);
    default: return r.qprior;
  }
}

// Half-step variants (all give the same bits):
//   k_half MODE 0: one lane (G = 1) or two lanes (G = 2) per pixel, scalar tap loops;
//   k_half MODE 1: one lane per pixel, row-pair f32x2 tap loops on the row-pair weight cache;
//   k_half_st:     row pairs plus the warp-collective staged source boxes (ncc_cost_warp).
// G = 1: two CTAs per SM with the weight cache (~90 KB each for a 13×13 window), four without it.
// G = 2: the two lanes of a pixel split the window rows, so each thread caches half the weights: four CTAs per SM.
// One half-step tile: CTA `cta` of the launch's flattened tile list, in phase `ph`, with dynamic shared memory sm.
template <int WR, int WS, bool CW, bool TEX, int G, int MODE>
__device__ __forceinline__ void half_tile(const PsRun& P, const HalfPhase& ph, int cta, float* sm) {
  constexpr int NT = PS_HALF_NT;
  constexpr int PW = half_pw(G);
  constexpr bool PAIRW = MODE >= 1;
  static_assert(MODE == 0 || (MODE == 1 && CW && G == 1 && WR != 0), "row pairs need the weight cache, one lane, a fixed window");
  const int wr = WR ? WR : P.wr, ws = WR ? WS : P.ws;
  const int wn = (2 * wr) / ws + 1;
  const int TW = half_tw(G, wr), TH = PS_HALF_PH + 2 * wr;
  float* tile = sm;
  float* wcache = sm + ((TW * TH + 31) & ~31);
  float* wvs = wcache + (CW ? ((wn + G - 1) / G) * wn * NT : 0);

  const int ii = find_item(P, cta);
  const PsItem& it = P.items[ii];
  if (!item_ok(P, it)) return;
  const int w = it.w, h = it.h;
  const int tiles_x = (w + PW - 1) / PW;
  const int tl = cta - it.tile0;
  const int x0 = (tl % tiles_x) * PW, y0 = (tl / tiles_x) * PS_HALF_PH;
  const PsLevel R = P.lv[it.view * P.nlevels + P.level];
  {
    const int ox = x0 - wr, oy = y0 - wr;
    for (int i = threadIdx.x; i < TW * TH; i += NT) {
      int tx = i % TW, ty = i / TW;
      int gx = ox + tx, gy = oy + ty;
      tile[i] = (gx >= 0 && gy >= 0 && gx < w && gy < h) ? R.img[gy * R.pitch + gx] : 0.f;
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gl = G == 2 ? (lane & 1) : 0;
  const int row = 2 * warp + (lane >> 4), col = G == 2 ? ((lane >> 1) & 7) : (lane & 15);
  const int y = y0 + row;
  const int x = x0 + 2 * col + ((y + ph.color) & 1);
  if (x >= w || y >= h) return;  // both lanes of a pixel leave together

  RefWin rw;
  rw.t = tile + (row + wr) * TW + (x - x0 + wr);
  rw.tw = TW;
  refwin_bounds(rw, tile, TW * TH, P);
  rw.wc = wcache + (PAIRW ? 2 * threadIdx.x : threadIdx.x);
  rw.g = gl;
  rw.pmask = G == 2 ? (3u << (lane & ~1)) : 0u;
  rw.wl = wcache + (wn & ~1) * wn * NT + threadIdx.x;
  float* wv = wvs + threadIdx.x;

  const PsView& vd = P.views[it.view];
  const PsPair* prs = P.pairs + (size_t)it.view * PS_MAXSRC;
  const PsLPair* lps = P.lpairs + ((size_t)it.view * P.nlevels + P.level) * PS_MAXSRC;
  const int nsrc = vd.nsrc;
  const long long base = it.off;
  const int pix = y * w + x;
  float4* pl = P.plane + base;
  const float3 ray = pixel_ray(R, x, y);

  float4 hyp[9];
  propagation_candidates(R, pl, P.cost + base, x, y, w, h, ray, hyp);

  // One NCC window of this pixel (the homography H is valid where hok).
  int nwin = 0;
  const RefStats rs = ref_stats<WR, WS, CW, NT, G, PAIRW>(P, rw);
  auto window = [&](const PsLevel& S, const float* H, bool hok) -> float {
    if constexpr (MODE == 1) {
      if (!hok || !ncc_begin(rs, S, H, (float)x, (float)y)) return 2.0f;
      nwin++;
      return ncc_window_lane<WR, WS, NT, TEX>(P, rw, rs, S, H, x, y);
    } else {
      return hok ? ncc_cost<WR, WS, CW, NT, TEX, G>(P, rw, rs, S, H, x, y, nwin) : 2.0f;
    }
  };

  // 2. View traversal: voting, weighting, aggregation.
  const int vprev = P.bview[base + pix];
  ViewAgg ag;
  agg_init(ag);
#pragma unroll 1
  for (int j = 0; j < nsrc; ++j) {
    const PsPair& pr = prs[j];
    const PsLPair lp = lps[j];
    const PsLevel S = P.lv[pr.src * P.nlevels + P.level];
    float m[9], gg[9];
    float prior;
    wv[j * NT] = 0.f;
    {
      float H[9];
      const bool ok = homography(R, lp, (float)x, (float)y, hyp[0], H);
      prior = view_prior(P, R, pr, H, ok, x, y, hyp[0], wr);
      if (!(prior > 0.f)) continue;
    }
#pragma unroll 1
    for (int i = 0; i < 9; ++i) {
      float H[9];
      const bool ok = homography(R, lp, (float)x, (float)y, hyp[i], H);
      const float mi = window(S, H, ok);
      const float gi = P.geometric ? fminf(geo_error(P, R, S, pr, x, y, hyp[i].w), P.gmax) : 0.f;
#pragma unroll
      for (int q = 0; q < 9; ++q)
        if (q == i) {
          m[q] = mi;
          gg[q] = gi;
        }
    }
    agg_source(P, ph.tau_good, ag, m, gg, prior, j, vprev, wv + j * NT);
  }
  float4 best;
  float bcost;
  agg_finish(ag, hyp, nsrc, wv, NT, best, bcost);

  // 3. Refinement, 6 hypotheses (patchmatch.cu:596-628), then 4. the coarse-scale candidate (:629-653).
  // A candidate's cost nm / den only grows as sources are added (every term wj·(mm + λ·g) is finite and ≥ 0, and
  // round-to-nearest addition and division by den > 0 are monotone), so once the partial cost reaches bcost the
  // candidate cannot be adopted (the test is cc < bcost) and its remaining windows are skipped: same decisions,
  // same bits.
  Refine rf;
  int nskip = 0;
  refine_prior(P, base + pix, rs.var, ray, rf);
  refine_draw(P, ph, vd, pix, ray, best, rf);
#pragma unroll 1
  for (int c = 0; c < rf.ncand; ++c) {
    const float4 cd = refine_candidate(rf, c);
    float cc;
    if (ag.den > 0.f) {
      float nm = 0.f;
      bool beaten = false;
#pragma unroll 1
      for (int j = 0; j < nsrc; ++j) {  // no break: the warp's lanes keep stepping through the sources together
        const float wj = wv[j * NT];
        if (!(wj > 0.f)) continue;
        beaten = beaten || nm / ag.den >= bcost;
        if (beaten) {
          nskip++;
          continue;
        }
        const PsPair& pr = prs[j];
        const PsLPair lp = lps[j];
        const PsLevel S = P.lv[pr.src * P.nlevels + P.level];
        float H[9];
        const bool hok = homography(R, lp, (float)x, (float)y, cd, H);
        const float mm = window(S, H, hok);
        const float g = P.geometric ? fminf(geo_error(P, R, S, pr, x, y, cd.w), P.gmax) : 0.f;
        nm += wj * (mm + P.lambda * g);
      }
      cc = beaten ? bcost : nm / ag.den;
    } else {
      cc = 2.f;
    }
    if (cc < bcost) {
      bcost = cc;
      best = cd;
    }
  }
  if (gl == 0) {
    pl[pix] = best;
    P.cost[base + pix] = bcost;
    P.bview[base + pix] = (unsigned char)ag.vbest;
  }
  count_windows(P, gl == 0 ? nwin : 0);
  count_skipped(P, gl == 0 ? nskip : 0);
}

template <int WR, int WS, bool CW, bool TEX, int G, int MODE = 0>
__global__ void __launch_bounds__(PS_HALF_NT, (CW && G == 1) ? 2 : 4) k_half(const __grid_constant__ PsRun P) {
  extern __shared__ float sm[];
  half_tile<WR, WS, CW, TEX, G, MODE>(P, launch_phase(P), blockIdx.x, sm);
}

// ================================================================================ persistent half step (PS_TUNE_PERSISTENT)
// Bounded wait of one thread until *ctr >= need (acquire at GPU scope, so the CTA's loads after the following barrier
// see the counted tiles' stores).  Gives up when another CTA has already given up (error word set) or after
// PS_QUEUE_SPIN_LIMIT polls, setting the error word; returns whether the count was reached.
__device__ __forceinline__ bool queue_wait(const PsRun& P, const unsigned* ctr, unsigned need) {
  for (unsigned spins = 0;; ++spins) {
    unsigned v, e;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(ctr) : "memory");
    if (v >= need) return true;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(e) : "l"(P.queue + 1) : "memory");
    if (e != 0u) return false;
    if (spins >= PS_QUEUE_SPIN_LIMIT) {
      atomicCAS(P.queue + 1, 0u, 1u);
      return false;
    }
    __nanosleep(256);
  }
}

// Every half step of a run in one launch.  Items (phase k, tile c) are handed out in the order k·ntiles + c from the
// queue counter, so all tiles of phase k precede those of phase k + 1; before a tile of phase k > 0 runs, its CTA
// waits until every tile of phase k - 1 of the same view is done (the tile reads the other colour's planes that
// phase k - 1 wrote, and overwrites planes that phase k - 1 read).  A CTA only dequeues when it is running and only
// waits on items dequeued before its own, so the smallest unfinished item never waits: the queue cannot deadlock,
// whatever the grid size.  When a wait gives up, the tile is skipped (its count is still added, so nothing waits on
// it) and the run reports PS_ETIMEOUT; every later wait returns at once.  The tiles compute exactly what the
// per-half-step launches compute, so the results are the same bits.
//
// A CTA that has seen phase k - 1 of a view complete (an acquire) needs no second wait for it: its later loads see
// those stores.  It remembers the last completed phase per view (s_seen), so a CTA waits about once per view and
// phase instead of once per tile.
template <int WR, int WS, bool TEX>
__global__ void __launch_bounds__(PS_HALF_NT, 2) k_half_q(const __grid_constant__ PsRun P) {
  extern __shared__ float sm[];
  __shared__ int s_item, s_go;
  __shared__ int s_seen[PS_MAX_ITEMS];
  const int total = P.ntiles * P.nphases;
  if (threadIdx.x < PS_MAX_ITEMS) s_seen[threadIdx.x] = -1;
  __syncthreads();
  for (;;) {
    if (threadIdx.x == 0) {
      const int i = (int)atomicAdd(P.queue, 1u);
      int go = 1;
      if (i < total) {
        const int k = i / P.ntiles, cta = i - k * P.ntiles;
        if (k > 0) {
          const int ii = find_item(P, cta);
          if (s_seen[ii] < k - 1 || P.qstall) {
            const int next = ii + 1 < P.nitems ? P.items[ii + 1].tile0 : P.ntiles;
            const unsigned need = (unsigned)(next - P.items[ii].tile0) + (P.qstall ? 1u : 0u);
            go = queue_wait(P, P.queue + 2 + (size_t)(k - 1) * P.nitems + ii, need) ? 1 : 0;
            if (go) s_seen[ii] = k - 1;
          }
        }
      }
      s_item = i;
      s_go = go;
    }
    __syncthreads();
    const int i = s_item;
    if (i >= total) return;
    const int k = i / P.ntiles, cta = i - k * P.ntiles;
    if (s_go) {
      const PsPhase& q = P.phases[k];
      half_tile<WR, WS, true, TEX, 1, 1>(P, HalfPhase{q.t, q.color, q.tau_good, q.eps, q.phi}, cta, sm);
    }
    __syncthreads();  // the tile's stores (and its reads of s_item) are done
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(P.queue + 2 + (size_t)k * P.nitems + find_item(P, cta), 1u);
    }
  }
}

// Staged-source half step.  One lane per pixel; a warp covers an 8 × 8 pixel block of the 32 × 8 tile.  Every
// window of every lane goes through ncc_cost_warp, which the whole warp calls together, so no lane leaves early
// (lanes outside the image work on a clamped pixel with every window inactive and write nothing) and the pixel's
// windows run as one job list with a single window call site: first the traversal jobs (source j, hypothesis i) in
// the reference's order, then the refinement jobs (candidate c, source j).  The arithmetic and the order of every
// sum are those of k_half, so the bits are the same.
//
// TMA (PS_TUNE_TMA): the reference tile and the source boxes arrive by 2-D tensor loads on mbarriers instead of the
// tile copy loop and the cp.async chunks.  The tile then starts tma_xo(wr) ≥ wr columns left of the CTA's first
// column (so its first element is 16-byte aligned) and reads the plane's zero border, padding and out-of-tensor zeros
// where the copy loop writes zeros outside the image: the same values.
__host__ __device__ constexpr int tma_xo(int wr) { return wr + ((PS_BORDER - wr) & 3); }
template <int WR, int WS, bool TEX, bool TMA>
__global__ void __launch_bounds__(PS_HALF_NT, 2) k_half_st(const __grid_constant__ PsRun P) {
  constexpr int NT = PS_HALF_NT;
  constexpr int wr = WR, wn = (2 * WR) / WS + 1;
  constexpr int XO = TMA ? tma_xo(WR) : WR;  // tile columns left of the CTA's first column
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(128) float sm[];
  __shared__ __align__(8) unsigned long long bars[1 + PS_HALF_NT / 32];
  const int TW = half_tw_staged(wr), TH = PS_HALF_PH + 2 * wr;
  static_assert(!TMA || PS_HALF_PW + tma_xo(WR) + WR <= half_tw_staged(WR), "TMA tile wider than the tile pitch");
  float* tile = sm;
  float* wcache = sm + ((TW * TH + 31) & ~31);
  float* wvs = wcache + wn * wn * NT;
  float* boxes = wvs + P.maxsrc * NT;

  const int ii = find_item(P, blockIdx.x);
  const PsItem& it = P.items[ii];
  if (!item_ok(P, it)) return;
  const int w = it.w, h = it.h;
  const int tiles_x = (w + PS_HALF_PW - 1) / PS_HALF_PW;
  const int tl = blockIdx.x - it.tile0;
  const int x0 = (tl % tiles_x) * PS_HALF_PW, y0 = (tl / tiles_x) * PS_HALF_PH;
  const PsLevel R = P.lv[it.view * P.nlevels + P.level];
  if constexpr (TMA) {
    // the tensor loads need 128-byte aligned destinations: the tile (the start of dynamic shared memory) and the
    // boxes (whole multiples of 128 bytes after it); otherwise nothing is loaded and the run fails (error word 3)
    if (((unsigned)__cvta_generic_to_shared(sm) & 127u) != 0u) {
      if (threadIdx.x == 0 && P.queue) atomicCAS(P.queue + 1, 0u, 3u);
      return;
    }
    const unsigned bar0 = (unsigned)__cvta_generic_to_shared(bars);
    if (threadIdx.x == 0) {
      for (int b = 0; b < 1 + PS_HALF_NT / 32; ++b) mbar_init(bar0 + 8u * b);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      fence_proxy_async();
      tma_load_2d((unsigned)__cvta_generic_to_shared(tile), tmap(P, it.view, 0), x0 - XO + PS_BORDER,
                  y0 - wr + PS_BORDER, bar0, (unsigned)(TW * TH * 4));
    }
    __syncthreads();  // barriers initialised
    mbar_wait(P, bar0, 0u);
  } else {
    const int ox = x0 - wr, oy = y0 - wr;
    for (int i = threadIdx.x; i < TW * TH; i += NT) {
      int tx = i % TW, ty = i / TW;
      int gx = ox + tx, gy = oy + ty;
      tile[i] = (gx >= 0 && gy >= 0 && gx < w && gy < h) ? R.img[gy * R.pitch + gx] : 0.f;
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int y = y0 + (lane >> 2);
  const HalfPhase ph = launch_phase(P);
  int x = x0 + 2 * (4 * warp + (lane & 3)) + ((y + ph.color) & 1);
  const bool live = x < w && y < h;
  y = min(y, h - 1);
  x = min(x, w - 1);
  float* box = boxes + warp * (PS_BOX_P * PS_BOX_H);
  BoxState bs{nullptr, 0, 0, (unsigned)__cvta_generic_to_shared(bars) + 8u * (1 + warp), 0u, 0, 0, 0, 0, 0, 0};

  RefWin rw;
  rw.t = tile + (y - y0 + wr) * TW + (x - x0 + XO);
  rw.tw = TW;
  refwin_bounds(rw, tile, TW * TH, P);
  rw.wc = wcache + 2 * threadIdx.x;
  rw.g = 0;
  rw.pmask = 0u;
  rw.wl = wcache + (wn & ~1) * wn * NT + threadIdx.x;
  float* wv = wvs + threadIdx.x;

  const PsView& vd = P.views[it.view];
  const PsPair* prs = P.pairs + (size_t)it.view * PS_MAXSRC;
  const PsLPair* lps = P.lpairs + ((size_t)it.view * P.nlevels + P.level) * PS_MAXSRC;
  const int nsrc = vd.nsrc;
  const long long base = it.off;
  const int pix = y * w + x;
  float4* pl = P.plane + base;
  const float3 ray = pixel_ray(R, x, y);
  const float fx = (float)x, fy = (float)y;

  float4 hyp[9];
  propagation_candidates(R, pl, P.cost + base, x, y, w, h, ray, hyp);
  int nwin = 0;
  const RefStats rs = ref_stats<WR, WS, true, NT, 1, true>(P, rw);
  const int vprev = P.bview[base + pix];
  Refine rf;
  refine_prior(P, base + pix, rs.var, ray, rf);

  const int nA = nsrc * 9;
  const int nB = (int)__reduce_max_sync(FULL, (unsigned)rf.ncand) * nsrc;
  ViewAgg ag;
  agg_init(ag);
  float m[9], gg[9];
  float prior = 0.f, nm = 0.f;
  int nskip = 0;
  bool use = false;
  float4 best = hyp[0];
  float bcost = 2.f;
#pragma unroll 1
  for (int k = 0;; ++k) {
    if (k == nA) {  // end of the traversal: aggregate, then the refinement draws
      agg_finish(ag, hyp, nsrc, wv, NT, best, bcost);
      refine_draw(P, ph, vd, pix, ray, best, rf);
    }
    if (k == nA + nB) break;
    const bool trav = k < nA;
    int j, i = 0, c = 0;
    if (trav) {
      j = k / 9;
      i = k - 9 * j;
    } else {
      c = (k - nA) / nsrc;
      j = (k - nA) - c * nsrc;
    }
    const PsPair& pr = prs[j];
    const PsLPair lp = lps[j];
    const PsLevel S = P.lv[pr.src * P.nlevels + P.level];
    float4 hv;
    bool act;
    float wj = 0.f;
    if (trav) {
      if (i == 0) {
        wv[j * NT] = 0.f;
        float H[9];
        const bool ok = homography(R, lp, fx, fy, hyp[0], H);
        prior = view_prior(P, R, pr, H, ok, x, y, hyp[0], wr);
        use = prior > 0.f && live;
      }
      hv = hyp[i];
      act = use;
    } else {
      hv = refine_candidate(rf, c);
      wj = wv[j * NT];
      // the candidate's partial cost already reaches bcost: its remaining windows cannot change the outcome
      act = c < rf.ncand && ag.den > 0.f && live && wj > 0.f;
      if (act && nm / ag.den >= bcost) {
        act = false;
        nskip++;
      }
    }
    float mv = 2.f;
    if (__any_sync(FULL, act)) {
      float H[9];
      const bool hok = homography(R, lp, fx, fy, hv, H);
      mv = ncc_cost_warp<WR, WS, NT, TEX, TMA>(P, rw, rs, S, pr.src, H, x, y, act && hok, nwin, box, bs);
    }
    if (trav) {
      const float gv = (P.geometric && use) ? fminf(geo_error(P, R, S, pr, x, y, hv.w), P.gmax) : 0.f;
#pragma unroll
      for (int q = 0; q < 9; ++q)
        if (q == i) {
          m[q] = mv;
          gg[q] = gv;
        }
      if (i == 8 && use) agg_source(P, ph.tau_good, ag, m, gg, prior, j, vprev, wv + j * NT);
    } else {
      if (act) {
        const float g = P.geometric ? fminf(geo_error(P, R, S, pr, x, y, hv.w), P.gmax) : 0.f;
        nm += wj * (mv + P.lambda * g);
      }
      if (j == nsrc - 1) {
        const float cc = ag.den > 0.f ? nm / ag.den : 2.f;
        if (c < rf.ncand && cc < bcost) {
          bcost = cc;
          best = hv;
        }
        nm = 0.f;
      }
    }
  }
  if (live) {
    pl[pix] = best;
    P.cost[base + pix] = bcost;
    P.bview[base + pix] = (unsigned char)ag.vbest;
  }
  count_windows(P, nwin);
  count_skipped(P, nskip);
  if (P.stage_count) {
    const unsigned c0 = __reduce_add_sync(FULL, (unsigned)bs.nstaged), c2 = __reduce_add_sync(FULL, (unsigned)bs.nbound);
    const unsigned c3 = __reduce_add_sync(FULL, (unsigned)bs.nwide), c4 = __reduce_add_sync(FULL, (unsigned)bs.ntall);
    const unsigned c5 = __reduce_add_sync(FULL, (unsigned)bs.nfew);
    if (lane == 0) {
      atomicAdd(P.stage_count, (unsigned long long)c0);
      atomicAdd(P.stage_count + 1, (unsigned long long)bs.nrestage);
      atomicAdd(P.stage_count + 2, (unsigned long long)c2);
      atomicAdd(P.stage_count + 3, (unsigned long long)c3);
      atomicAdd(P.stage_count + 4, (unsigned long long)c4);
      atomicAdd(P.stage_count + 5, (unsigned long long)c5);
    }
  }
}

// ================================================================================ run start / evaluate (patchmatch.cu:661-692)
// Top-K mean cost (patchmatch.cu:327-345).
template <int WR, int WS, bool CW, int NT, bool TEX = false>
__device__ float topk_cost(const PsRun& P, const RefWin& rw, const RefStats& rs, const PsLevel& R, const PsPair* prs,
                           const PsLPair* lps, int nsrc, int x, int y, float4 h, int& nwin) {
  float b0 = 1e30f, b1 = 1e30f, b2 = 1e30f;
#pragma unroll 1
  for (int j = 0; j < nsrc; ++j) {
    const PsPair& pr = prs[j];
    const PsLPair lp = lps[j];
    const PsLevel S = P.lv[pr.src * P.nlevels + P.level];
    float g = 0.f;
    float c = pair_cost<WR, WS, CW, NT, TEX>(P, rw, rs, R, S, pr, lp, x, y, h, &g, nwin);
    if (P.geometric) c += P.lambda * g;
    if (c < b0) {
      b2 = b1;
      b1 = b0;
      b0 = c;
    } else if (c < b1) {
      b2 = b1;
      b1 = c;
    } else if (c < b2) {
      b2 = c;
    }
  }
  const int k = min(P.topk, nsrc);
  float s = b0;
  if (k >= 2) s += b1;
  if (k >= 3) s += b2;
  return k > 0 ? s / (float)k : 2.0f;
}

// Loads the 32 × 4 reference tile of an evaluate/filter CTA; returns false for threads outside the image.
struct EvalCtx {
  int x, y, w, h;
  const PsItem* it;
  PsLevel R;
};
__device__ __forceinline__ bool eval_tile(const PsRun& P, float* tile, int wr, EvalCtx& e) {
  const int ii = find_item(P, blockIdx.x);
  const PsItem& it = P.items[ii];
  if (!item_ok(P, it)) return false;
  e.it = &it;
  e.w = it.w;
  e.h = it.h;
  const int tiles_x = (it.w + PS_EVAL_PW - 1) / PS_EVAL_PW;
  const int tl = blockIdx.x - it.tile0;
  const int x0 = (tl % tiles_x) * PS_EVAL_PW, y0 = (tl / tiles_x) * PS_EVAL_PH;
  e.R = P.lv[it.view * P.nlevels + P.level];
  const int TW = PS_EVAL_PW + 2 * wr, TH = PS_EVAL_PH + 2 * wr;
  const int ox = x0 - wr, oy = y0 - wr;
  for (int i = threadIdx.x; i < TW * TH; i += PS_EVAL_NT) {
    int tx = i % TW, ty = i / TW;
    int gx = ox + tx, gy = oy + ty;
    tile[i] = (gx >= 0 && gy >= 0 && gx < it.w && gy < it.h) ? e.R.img[gy * e.R.pitch + gx] : 0.f;
  }
  __syncthreads();
  e.x = x0 + (threadIdx.x & 31);
  e.y = y0 + (threadIdx.x >> 5);
  return e.x < it.w && e.y < it.h;
}

// TEX: the source samples through the planes' texture gathers (same bits as the plane loads).
template <int WR, int WS, bool CW, bool TEX>
__global__ void __launch_bounds__(PS_EVAL_NT, 2) k_eval(const __grid_constant__ PsRun P) {
  constexpr int NT = PS_EVAL_NT;
  extern __shared__ float sm[];
  const int wr = WR ? WR : P.wr;
  const int TW = PS_EVAL_PW + 2 * wr, TH = PS_EVAL_PH + 2 * wr;
  EvalCtx e;
  if (!eval_tile(P, sm, wr, e)) return;
  const int x = e.x, y = e.y;
  RefWin rw;
  {
    const int tiles_x = (e.w + PS_EVAL_PW - 1) / PS_EVAL_PW;
    const int tl = blockIdx.x - e.it->tile0;
    const int x0 = (tl % tiles_x) * PS_EVAL_PW, y0 = (tl / tiles_x) * PS_EVAL_PH;
    rw.t = sm + (y - y0 + wr) * TW + (x - x0 + wr);
  }
  rw.tw = TW;
  refwin_bounds(rw, sm, TW * TH, P);
  rw.wc = sm + ((TW * TH + 31) & ~31) + threadIdx.x;
  const PsItem& it = *e.it;
  const PsView& vd = P.views[it.view];
  const PsPair* prs = P.pairs + (size_t)it.view * PS_MAXSRC;
  const PsLPair* lps = P.lpairs + ((size_t)it.view * P.nlevels + P.level) * PS_MAXSRC;
  const int pix = y * e.w + x;
  const long long base = it.off;
  const float3 ray = pixel_ray(e.R, x, y);
  float4 h = P.plane[base + pix];
  if (P.mode == 1 && P.random_init) {
    u64 st = rng_state(P.seed, vd.key, P.level, P.run_id, 0xFFFF, 0, (u64)pix);
    const float d = random_depth(st, vd.dmin, vd.dmax);
    const float3 n = random_normal(st, ray);
    h = make_float4(n.x, n.y, n.z, d);
    if (P.proposal) {  // learned init: a proposed plane (d > 0) replaces the random draw; elsewhere the draw stays
      const float4 q = P.proposal[base + pix];
      if (q.w > 0.f) h = q;
    }
    P.plane[base + pix] = h;
  }
  float c = 2.f;
  int nwin = 0;
  if (h.w > 0.f) {
    const RefStats rs = ref_stats<WR, WS, CW, NT>(P, rw);
    c = topk_cost<WR, WS, CW, NT, TEX>(P, rw, rs, e.R, prs, lps, vd.nsrc, x, y, h, nwin);
  }
  P.cost[base + pix] = c;
  if (P.mode == 1) P.bview[base + pix] = 255;
  count_windows(P, nwin);
}

// ================================================================================ plane sweep (learned proposal input)
// Cost volume of one view for the proposal network (no reference counterpart).  PS_SWEEP_PLANES planes with the
// normal P.sweep_n (fronto-parallel (0, 0, -1) unless the caller set one, e.g. the world's up direction in the camera
// frame) through inverse depths i_k = 1/dmax + (2k+1)/64 · (1/dmin - 1/dmax) (bin centres) at the pixel; the cost of a
// plane is the mean over the first min(2, nsrc) sources of the NCC cost 1 - ρ (the same window statistics, homography
// and NCC as the half step, window radius wr and step P.sweep_ws), 2 where the homography fails.  Output per pixel,
// bf16 (round to nearest even): [image, cost_0 … cost_31, 0 × 15] at netin[(y · netin_pitch + x) · 48].
__device__ __forceinline__ unsigned short bf16_bits(float v) {
  const __nv_bfloat16 b = __float2bfloat16_rn(v);
  return *reinterpret_cast<const unsigned short*>(&b);
}

template <int WR, int WS, bool TEX>
__global__ void __launch_bounds__(PS_EVAL_NT, 2) k_sweep(const __grid_constant__ PsRun P) {
  constexpr int NT = PS_EVAL_NT;
  extern __shared__ float sm[];
  const int wr = WR ? WR : P.wr;
  const int TW = PS_EVAL_PW + 2 * wr, TH = PS_EVAL_PH + 2 * wr;
  EvalCtx e;
  if (!eval_tile(P, sm, wr, e)) return;
  const int x = e.x, y = e.y;
  RefWin rw;
  {
    const int tiles_x = (e.w + PS_EVAL_PW - 1) / PS_EVAL_PW;
    const int tl = blockIdx.x - e.it->tile0;
    const int x0 = (tl % tiles_x) * PS_EVAL_PW, y0 = (tl / tiles_x) * PS_EVAL_PH;
    rw.t = sm + (y - y0 + wr) * TW + (x - x0 + wr);
  }
  rw.tw = TW;
  refwin_bounds(rw, sm, TW * TH, P);
  rw.wc = sm + ((TW * TH + 31) & ~31) + threadIdx.x;
  const PsView& vd = P.views[e.it->view];
  const PsLPair* lps = P.lpairs + ((size_t)e.it->view * P.nlevels + P.level) * PS_MAXSRC;
  const PsPair* prs = P.pairs + (size_t)e.it->view * PS_MAXSRC;
  const int nuse = min(vd.nsrc, 2);
  const RefStats rs = ref_stats<WR, WS, true, NT>(P, rw);
  const float inear = 1.0f / vd.dmin, ifar = 1.0f / vd.dmax;
  unsigned short* out = P.netin + ((long long)y * P.netin_pitch + x) * PS_NET_CH_IN;
  out[0] = bf16_bits(tile_at(rw, rw.t));
  int nwin = 0;
#pragma unroll 1
  for (int k = 0; k < PS_SWEEP_PLANES; ++k) {
    const float id = fmaf((float)(2 * k + 1) * (1.0f / 64.0f), inear - ifar, ifar);
    const float4 h = make_float4(P.sweep_n[0], P.sweep_n[1], P.sweep_n[2], 1.0f / id);
    float c = 0.0f;
#pragma unroll 1
    for (int j = 0; j < nuse; ++j) {
      const PsLevel S = P.lv[prs[j].src * P.nlevels + P.level];
      float H[9];
      c += homography(e.R, lps[j], (float)x, (float)y, h, H)
               ? ncc_cost<WR, WS, true, NT, TEX>(P, rw, rs, S, H, x, y, nwin)
               : 2.0f;
    }
    c = nuse == 2 ? c * 0.5f : (nuse == 1 ? c : 2.0f);
    out[1 + k] = bf16_bits(c);
  }
#pragma unroll
  for (int k = 1 + PS_SWEEP_PLANES; k < PS_NET_CH_IN; ++k) out[k] = 0;
  count_windows(P, nwin);
}

// ================================================================================ final readout (patchmatch.cu:695-737)
template <int WR, int WS, bool CW, bool TEX>
__global__ void __launch_bounds__(PS_EVAL_NT, 2) k_filter(const __grid_constant__ PsRun P) {
  constexpr int NT = PS_EVAL_NT;
  extern __shared__ float sm[];
  const int wr = WR ? WR : P.wr;
  const int TW = PS_EVAL_PW + 2 * wr, TH = PS_EVAL_PH + 2 * wr;
  EvalCtx e;
  if (!eval_tile(P, sm, wr, e)) return;
  const int x = e.x, y = e.y;
  const PsItem& it = *e.it;
  RefWin rw;
  {
    const int tiles_x = (e.w + PS_EVAL_PW - 1) / PS_EVAL_PW;
    const int tl = blockIdx.x - it.tile0;
    const int x0 = (tl % tiles_x) * PS_EVAL_PW, y0 = (tl / tiles_x) * PS_EVAL_PH;
    rw.t = sm + (y - y0 + wr) * TW + (x - x0 + wr);
  }
  rw.tw = TW;
  refwin_bounds(rw, sm, TW * TH, P);
  rw.wc = sm + ((TW * TH + 31) & ~31) + threadIdx.x;
  const PsView& vd = P.views[it.view];
  const PsPair* prs = P.pairs + (size_t)it.view * PS_MAXSRC;
  const PsLPair* lps = P.lpairs + ((size_t)it.view * P.nlevels + P.level) * PS_MAXSRC;
  const int pix = y * e.w + x;
  const long long base = it.off;
  const float4 h = P.plane[base + pix];
  int count = 0;
  int nwin = 0;
  if (h.w > 0.f) {
    const RefStats rs = ref_stats<WR, WS, CW, NT>(P, rw);
    const float3 ray = pixel_ray(e.R, x, y);
    const float3 X = make_float3(ray.x * h.w, ray.y * h.w, h.w);
    const float lx = sqrtf(dot3(X, X));
#pragma unroll 1
    for (int j = 0; j < vd.nsrc; ++j) {
      const PsPair& pr = prs[j];
      const PsLevel S = P.lv[pr.src * P.nlevels + P.level];
      const float3 Sv = make_float3(pr.c[0] - X.x, pr.c[1] - X.y, pr.c[2] - X.z);
      const float ls = sqrtf(dot3(Sv, Sv));
      if (!(ls > 0.f)) continue;
      const float cost = -dot3(Sv, X) / (ls * lx);
      if (cost > P.cos_filter_tri) continue;
      const float cphi = dot3(Sv, make_float3(h.x, h.y, h.z)) / ls;
      if (cphi <= 0.f) continue;
      float H[9];
      const PsLPair lp = lps[j];
      if (!homography(e.R, lp, (float)x, (float)y, h, H)) continue;
      const float m = ncc_cost<WR, WS, CW, NT, TEX>(P, rw, rs, S, H, x, y, nwin);
      const float ee = P.ncc_norm * m_exp(-m * m * P.inv2ncc);
      if (ee / (ee + 0.5f) < P.q_min) continue;
      if (geo_error(P, e.R, S, pr, x, y, h.w) > P.filter_gmax) continue;
      count++;
    }
  }
  P.count[base + pix] = (unsigned char)min(count, 255);
  count_windows(P, nwin);
}

// Simple kernels: CTA of 32 × 8 threads, tiles flattened like the others.
struct SimpleCtx {
  int x, y;
  const PsItem* it;
};
__device__ __forceinline__ bool simple_px(const PsRun& P, SimpleCtx& c) {
  const int ii = find_item(P, blockIdx.x);
  const PsItem& it = P.items[ii];
  if (!item_ok(P, it)) return false;
  const int tiles_x = (it.w + PS_SIMPLE_BX - 1) / PS_SIMPLE_BX;
  const int tl = blockIdx.x - it.tile0;
  c.x = (tl % tiles_x) * PS_SIMPLE_BX + (int)threadIdx.x;
  c.y = (tl / tiles_x) * PS_SIMPLE_BY + (int)threadIdx.y;
  c.it = &it;
  return c.x < it.w && c.y < it.h;
}

// ================================================================================ joint bilateral upsampling (patchmatch.cu:741-801)
// Input: level-1 planes at P.prior + item.aux; output: level planes (cost reset to 2).
__global__ void __launch_bounds__(256) k_upsample(const __grid_constant__ PsRun P) {
  SimpleCtx c;
  if (!simple_px(P, c)) return;
  const PsItem& it = *c.it;
  const int x = c.x, y = c.y;
  const PsLevel R = P.lv[it.view * P.nlevels + P.level];
  const PsLevel L = P.lv[it.view * P.nlevels + P.level - 1];
  const float4* low = P.prior + it.aux;
  const float3 rp = pixel_ray(R, x, y);
  const float ip = R.img[y * R.pitch + x];
  const float px = ((float)x - 0.5f) * 0.5f, py = ((float)y - 0.5f) * 0.5f;
  const int qx0 = (int)roundf(px), qy0 = (int)roundf(py);
  float sw = 0.f, sd = 0.f;
  float3 sn = make_float3(0.f, 0.f, 0.f);
  float nd = 1e30f, ndep = 0.f;
  float3 nn = make_float3(0.f, 0.f, 0.f);
  for (int qy = qy0 - 2; qy <= qy0 + 2; ++qy) {
    if (qy < 0 || qy >= L.h) continue;
    for (int qx = qx0 - 2; qx <= qx0 + 2; ++qx) {
      if (qx < 0 || qx >= L.w) continue;
      const float4 q = low[qy * L.w + qx];
      if (!(q.w > 0.f)) continue;
      const float3 n = make_float3(q.x, q.y, q.z);
      const float den = dot3(n, rp);
      if (!(den < -1e-6f)) continue;
      const float d = q.w * dot3(n, pixel_ray(L, qx, qy)) / den;
      if (!(d > 0.f) || !isfinite(d)) continue;
      const float ds = ((float)qx - px) * ((float)qx - px) + ((float)qy - py) * ((float)qy - py);
      if (ds < nd) {
        nd = ds;
        ndep = d;
        nn = n;
      }
      const float iq = L.img[qy * L.pitch + qx];
      const float wgt = m_exp(-ds * P.up_inv2s - (ip - iq) * (ip - iq) * P.up_inv2c);
      sw += wgt;
      sd += wgt * d;
      sn.x += wgt * n.x;
      sn.y += wgt * n.y;
      sn.z += wgt * n.z;
    }
  }
  float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
  float d = 0.f;
  float3 n = make_float3(0.f, 0.f, 0.f);
  bool ok = false;
  if (sw > 1e-12f) {
    d = sd / sw;
    n = sn;
    ok = true;
  } else if (nd < 1e29f) {
    d = ndep;
    n = nn;
    ok = true;
  }
  if (ok && dot3(n, n) > 1e-24f) {
    n = nrm3(n);
    if (dot3(n, rp) >= 0.f) n = make_float3(-n.x, -n.y, -n.z);
    out = make_float4(n.x, n.y, n.z, d);
  }
  P.plane[it.off + y * it.w + x] = out;
  P.cost[it.off + y * it.w + x] = 2.f;
}

// ================================================================================ 5×5 median plane filter (patchmatch.cu:805-849)
// Input: planes at P.prior + item.aux (same level); output: P.plane at item.off.
__global__ void __launch_bounds__(256) k_median(const __grid_constant__ PsRun P) {
  SimpleCtx c;
  if (!simple_px(P, c)) return;
  const PsItem& it = *c.it;
  const int x = c.x, y = c.y, w = it.w, h = it.h;
  const PsLevel R = P.lv[it.view * P.nlevels + P.level];
  const float4* in = P.prior + it.aux;
  const float4 self = in[y * w + x];
  if (!(self.w > 0.f)) {
    P.plane[it.off + y * w + x] = self;
    return;
  }
  const float3 rp = pixel_ray(R, x, y);
  float ds[25];
  int qs[25];
  int cnt = 0;
  for (int qy = max(y - 2, 0); qy < min(y + 3, h); ++qy) {
    for (int qx = max(x - 2, 0); qx < min(x + 3, w); ++qx) {
      const float4 q = in[qy * w + qx];
      if (!(q.w > 0.f)) continue;
      const float3 n = make_float3(q.x, q.y, q.z);
      const float den = dot3(n, rp);
      if (!(den < -1e-6f)) continue;
      const float d = q.w * dot3(n, pixel_ray(R, qx, qy)) / den;
      if (!(d > 0.f) || !isfinite(d)) continue;
      const int qi = qy * w + qx;
      int k = cnt++;
      while (k > 0 && (ds[k - 1] > d || (ds[k - 1] == d && qs[k - 1] > qi))) {
        ds[k] = ds[k - 1];
        qs[k] = qs[k - 1];
        --k;
      }
      ds[k] = d;
      qs[k] = qi;
    }
  }
  float4 out = self;
  if (cnt > 0) {
    const int m = (cnt - 1) / 2;
    const float4 q = in[qs[m]];
    out = make_float4(q.x, q.y, q.z, ds[m]);
  }
  P.plane[it.off + y * w + x] = out;
}

// ================================================================================ helpers
// Snapshot capture: depth channel of the resident planes into the snapshot buffer (item.aux = snapshot offset).
__global__ void __launch_bounds__(256) k_snapshot(const __grid_constant__ PsRun P, float* snap) {
  SimpleCtx c;
  if (!simple_px(P, c)) return;
  const PsItem& it = *c.it;
  const int pix = c.y * it.w + c.x;
  snap[it.aux + pix] = P.plane[it.off + pix].w;
}

// Readout threshold (crates/dense/src/densify.rs:441-454): depth/normal zeroed where count < need.
__global__ void __launch_bounds__(256) k_readout(const __grid_constant__ PsRun P, float4* out) {
  SimpleCtx c;
  if (!simple_px(P, c)) return;
  const PsItem& it = *c.it;
  const int pix = c.y * it.w + c.x;
  const int nsrc = P.views[it.view].nsrc;
  int need = min(P.need_min, nsrc);
  if (need < 1) need = 1;
  const float4 q = P.plane[it.off + pix];
  const bool keep = q.w > 0.f && (int)P.count[it.off + pix] >= need;
  out[it.off + pix] = keep ? q : make_float4(0.f, 0.f, 0.f, 0.f);
}

// FP64 homography setup A = K_j R K^-1, b = K_j t for every (view, level, source) (crates/cuda/src/patchmatch.rs:132-151).
// One thread per (view, level, source); r/t come from pairs_f64 when given (15 doubles per source), else from the
// f32 pair table.
__global__ void k_setup_lpairs(const PsLevel* lv, const PsPair* pairs, const double* pairs64, const int* has64,
                               PsLPair* out, int nviews, int nlevels) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nviews * nlevels * PS_MAXSRC) return;
  const int j = idx % PS_MAXSRC;
  const int l = (idx / PS_MAXSRC) % nlevels;
  const int v = idx / (PS_MAXSRC * nlevels);
  const PsPair& pr = pairs[v * PS_MAXSRC + j];
  PsLPair o;
  for (int k = 0; k < 9; ++k) o.A[k] = 0.f;
  for (int k = 0; k < 3; ++k) o.b[k] = 0.f;
  if (pr.src >= 0) {
    const PsLevel& R = lv[v * nlevels + l];
    const PsLevel& J = lv[pr.src * nlevels + l];
    double r[9], t[3];
    if (has64[v]) {
      const double* p = pairs64 + ((size_t)v * PS_MAXSRC + j) * 15;
      for (int k = 0; k < 9; ++k) r[k] = p[k];
      for (int k = 0; k < 3; ++k) t[k] = p[9 + k];
    } else {
      for (int k = 0; k < 9; ++k) r[k] = (double)pr.r[k];
      for (int k = 0; k < 3; ++k) t[k] = (double)pr.t[k];
    }
    const double fx = R.fx, fy = R.fy, cx = R.cx, cy = R.cy;
    const double kinv[3][3] = {{1.0 / fx, 0.0, -cx / fx}, {0.0, 1.0 / fy, -cy / fy}, {0.0, 0.0, 1.0}};
    const double kj[3][3] = {{(double)J.fx, 0.0, (double)J.cx}, {0.0, (double)J.fy, (double)J.cy}, {0.0, 0.0, 1.0}};
    double kr[3][3];
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) kr[i][k] = kj[i][0] * r[0 * 3 + k] + kj[i][1] * r[1 * 3 + k] + kj[i][2] * r[2 * 3 + k];
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) o.A[i * 3 + k] = (float)(kr[i][0] * kinv[0][k] + kr[i][1] * kinv[1][k] + kr[i][2] * kinv[2][k]);
    for (int i = 0; i < 3; ++i) o.b[i] = (float)(kj[i][0] * t[0] + kj[i][1] * t[1] + kj[i][2] * t[2]);
  }
  out[idx] = o;
}

// Exhaustive check of m_rcp against the correctly rounded reciprocal (__frcp_rn): x = (1 + i/2^23)·2^e for every
// significand i (blockIdx.x·256 + threadIdx.x < 2^23) and exponent e = e_lo + blockIdx.y.  Counts mismatches and keeps
// the first 8 arguments that differ.
__global__ void __launch_bounds__(256) k_rcp_check(int e_lo, unsigned long long* bad, unsigned* first) {
  const unsigned i = blockIdx.x * 256u + threadIdx.x;
  if (i >= (1u << 23)) return;
  const unsigned bits = ((unsigned)(127 + e_lo + (int)blockIdx.y) << 23) | i;
  const float x = __uint_as_float(bits);
  if (__float_as_uint(m_rcp(x)) != __float_as_uint(__frcp_rn(x))) {
    const unsigned long long k = atomicAdd(bad, 1ull);
    if (k < 8) first[k] = bits;
  }
}

// FP32 throughput probe: 8 independent FFMA chains per thread, register resident.
__global__ void __launch_bounds__(256) k_fp32_probe(float* out, int iters, float a, float b) {
  float v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = (float)(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = fmaf(v[k], a, b);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += v[k];
  if (s == 12345.678f) out[blockIdx.x] = s;  // keeps the loop alive
}

// ================================================================================ launchers
#define PS_SPECS(X) X(5, 1) X(6, 1) X(5, 2) X(3, 1)

static int g_prop_ready = 0;

static cudaError_t init_constants() {
  if (g_prop_ready) return cudaSuccess;
  int2 h[72];
  const int V[7][2] = {{0, -1}, {-1, -2}, {1, -2}, {-2, -3}, {2, -3}, {-3, -4}, {3, -4}};
  int n = 0;
  for (int r = 0; r < 8; ++r) {
    const int dir = r & 3;
    const bool strip = r >= 4;
    const int cnt = strip ? 11 : 7;
    for (int k = 0; k < cnt; ++k) {
      int dx = strip ? 0 : V[k][0], dy = strip ? -(3 + 2 * k) : V[k][1];
      for (int q = 0; q < dir; ++q) {
        int t = dx;
        dx = -dy;
        dy = t;
      }
      h[n++] = make_int2(dx, dy);
    }
  }
  cudaError_t e = cudaMemcpyToSymbol(c_prop, h, sizeof h);
  if (e == cudaSuccess) g_prop_ready = 1;
  return e;
}

size_t half_smem(int wr, int ws, bool cw, int maxsrc, int G, int mode) {
  const int wn = (2 * wr) / ws + 1;
  const int TW = mode == 2 ? half_tw_staged(wr) : half_tw(G, wr), TH = PS_HALF_PH + 2 * wr;
  size_t f = ((TW * TH + 31) & ~31) + (cw ? (size_t)((wn + G - 1) / G) * wn * PS_HALF_NT : 0) +
             (size_t)maxsrc * PS_HALF_NT + (mode == 2 ? (size_t)(PS_HALF_NT / 32) * PS_BOX_P * PS_BOX_H : 0);
  return f * sizeof(float);
}
size_t eval_smem(int wr, int ws, bool cw) {
  const int wn = (2 * wr) / ws + 1;
  const int TW = PS_EVAL_PW + 2 * wr, TH = PS_EVAL_PH + 2 * wr;
  size_t f = ((TW * TH + 31) & ~31) + (cw ? (size_t)wn * wn * PS_EVAL_NT : 0);
  return f * sizeof(float);
}

// Whether the weight cache fits (<= 200 KB of shared memory per CTA with the largest source count).
static bool use_cache(int wr, int ws) { return half_smem(wr, ws, true, PS_MAXSRC, 1, 0) <= 200 * 1024; }

template <typename K>
static cudaError_t launch(K kern, int ncta, int nt, size_t smem, cudaStream_t st, const PsRun& P) {
  static_assert(sizeof(PsRun) < 32000, "kernel parameter block too large");
  if (ncta <= 0) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<ncta, nt, smem, st>>>(P);
  return cudaGetLastError();
}

// Half-step mode of a tuning word: 2 = staged source boxes (PS_TUNE_STAGED), 1 = row-pair loops (PS_TUNE_ROW_PAIRS),
// 0 = scalar loops.  The row-pair modes need one lane per pixel, the weight cache and a compiled window; otherwise the
// scalar kernel runs (same bits).
static int half_mode(unsigned tuning, int wr, int ws) {
  if (!(tuning & 0x18u) || (tuning & 0x1u) || !use_cache(wr, ws)) return 0;
  bool compiled = false;
#define PS_CASE(a, b) compiled = compiled || (wr == a && ws == b);
  PS_SPECS(PS_CASE)
#undef PS_CASE
  if (!compiled) return 0;
  return (tuning & 0x10u) ? 2 : 1;
}

// Lanes per pixel of the half-step kernel for a tuning word (PS_TUNE_ONE_LANE or a row-pair mode selects 1, default 2).
int half_lanes(unsigned tuning) { return (tuning & 0x1Cu) ? 1 : 2; }

template <int A, int B, int G>
static cudaError_t launch_half_g(const PsRun& P, bool cw, bool tex, size_t smem, cudaStream_t st) {
  if (cw) return tex ? launch(k_half<A, B, true, true, G>, P.ntiles, PS_HALF_NT, smem, st, P)
                     : launch(k_half<A, B, true, false, G>, P.ntiles, PS_HALF_NT, smem, st, P);
  return tex ? launch(k_half<A, B, false, true, G>, P.ntiles, PS_HALF_NT, smem, st, P)
             : launch(k_half<A, B, false, false, G>, P.ntiles, PS_HALF_NT, smem, st, P);
}
template <int A, int B>
static cudaError_t launch_half_pairs(const PsRun& P, int mode, bool tex, size_t smem, cudaStream_t st) {
  if (mode == 2) {
    if (P.tmaps) return tex ? launch(k_half_st<A, B, true, true>, P.ntiles, PS_HALF_NT, smem, st, P)
                            : launch(k_half_st<A, B, false, true>, P.ntiles, PS_HALF_NT, smem, st, P);
    return tex ? launch(k_half_st<A, B, true, false>, P.ntiles, PS_HALF_NT, smem, st, P)
               : launch(k_half_st<A, B, false, false>, P.ntiles, PS_HALF_NT, smem, st, P);
  }
  return tex ? launch(k_half<A, B, true, true, 1, 1>, P.ntiles, PS_HALF_NT, smem, st, P)
             : launch(k_half<A, B, true, false, 1, 1>, P.ntiles, PS_HALF_NT, smem, st, P);
}

// Whether the persistent kernel runs a run's half steps for this tuning word and window: the row-pair mode with
// PS_TUNE_PERSISTENT.
bool half_run_ok(unsigned tuning, int wr, int ws) { return (tuning & 0x20u) && half_mode(tuning, wr, ws) == 1; }

// The persistent half step: as many CTAs as fit on the device at once (or fewer when there are fewer items).
template <int A, int B>
static cudaError_t launch_half_q(const PsRun& P, bool tex, size_t smem, cudaStream_t st) {
  void (*kern)(PsRun) = tex ? k_half_q<A, B, true> : k_half_q<A, B, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, PS_HALF_NT, smem)) != cudaSuccess) return e;
  const long long total = (long long)P.ntiles * P.nphases;
  const long long grid = std::min<long long>(total, (long long)std::max(per, 1) * sms);
  if (grid <= 0) return cudaSuccess;
  kern<<<(int)grid, PS_HALF_NT, smem, st>>>(P);
  return cudaGetLastError();
}

// Every half step of P's phase table in one launch (half_run_ok must hold); P.queue must be zeroed on the stream.
cudaError_t launch_half_run(const PsRun& P, unsigned tuning, cudaStream_t st) {
  cudaError_t e = init_constants();
  if (e != cudaSuccess) return e;
  if (!half_run_ok(tuning, P.wr, P.ws) || !P.queue || P.nphases < 1 || P.nphases > PS_MAX_PHASES)
    return cudaErrorInvalidValue;
  const bool tex = (tuning & 0x2u) != 0;
  const size_t smem = half_smem(P.wr, P.ws, true, P.maxsrc, 1, 1);
#define PS_CASE(a, b) \
  if (P.wr == a && P.ws == b) return launch_half_q<a, b>(P, tex, smem, st);
  PS_SPECS(PS_CASE)
#undef PS_CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_half(const PsRun& P, unsigned tuning, cudaStream_t st) {
  cudaError_t e = init_constants();
  if (e != cudaSuccess) return e;
  const bool tex = (tuning & 0x2u) != 0;
  const int mode = half_mode(tuning, P.wr, P.ws);
  if (mode != 0) {
    const size_t smem = half_smem(P.wr, P.ws, true, P.maxsrc, 1, mode);
#define PS_CASE(a, b) \
    if (P.wr == a && P.ws == b) return launch_half_pairs<a, b>(P, mode, tex, smem, st);
    PS_SPECS(PS_CASE)
#undef PS_CASE
  }
  const bool cw = use_cache(P.wr, P.ws) && !(tuning & 0x1u);
  const int G = half_lanes(tuning);
  const size_t smem = half_smem(P.wr, P.ws, cw, P.maxsrc, G, 0);
#define PS_CASE(a, b)                                                                \
  if (P.wr == a && P.ws == b)                                                        \
    return G == 2 ? launch_half_g<a, b, 2>(P, cw, tex, smem, st) : launch_half_g<a, b, 1>(P, cw, tex, smem, st);
  PS_SPECS(PS_CASE)
#undef PS_CASE
  return G == 2 ? launch_half_g<0, 1, 2>(P, cw, tex, smem, st) : launch_half_g<0, 1, 1>(P, cw, tex, smem, st);
}

// tex: the session built texture objects for its planes (PS_TUNE_TEX_GATHER); the specialised windows then sample
// through them, the generic kernels keep the plane loads.
cudaError_t launch_eval(const PsRun& P, bool tex, cudaStream_t st) {
  const bool cw = use_cache(P.wr, P.ws);
  const size_t smem = eval_smem(P.wr, P.ws, cw);
#define PS_CASE(a, b)                                                                                  \
  if (P.wr == a && P.ws == b)                                                                          \
    return tex ? launch(k_eval<a, b, true, true>, P.ntiles, PS_EVAL_NT, smem, st, P)                   \
               : launch(k_eval<a, b, true, false>, P.ntiles, PS_EVAL_NT, smem, st, P);
  PS_SPECS(PS_CASE)
#undef PS_CASE
  if (cw) return launch(k_eval<0, 1, true, false>, P.ntiles, PS_EVAL_NT, smem, st, P);
  return launch(k_eval<0, 1, false, false>, P.ntiles, PS_EVAL_NT, smem, st, P);
}

cudaError_t launch_filter(const PsRun& P, bool tex, cudaStream_t st) {
  const bool cw = use_cache(P.wr, P.ws);
  const size_t smem = eval_smem(P.wr, P.ws, cw);
#define PS_CASE(a, b)                                                                                  \
  if (P.wr == a && P.ws == b)                                                                          \
    return tex ? launch(k_filter<a, b, true, true>, P.ntiles, PS_EVAL_NT, smem, st, P)                 \
               : launch(k_filter<a, b, true, false>, P.ntiles, PS_EVAL_NT, smem, st, P);
  PS_SPECS(PS_CASE)
#undef PS_CASE
  if (cw) return launch(k_filter<0, 1, true, false>, P.ntiles, PS_EVAL_NT, smem, st, P);
  return launch(k_filter<0, 1, false, false>, P.ntiles, PS_EVAL_NT, smem, st, P);
}

cudaError_t launch_upsample(const PsRun& P, cudaStream_t st) {
  if (P.ntiles <= 0) return cudaSuccess;
  k_upsample<<<P.ntiles, dim3(PS_SIMPLE_BX, PS_SIMPLE_BY), 0, st>>>(P);
  return cudaGetLastError();
}
cudaError_t launch_median(const PsRun& P, cudaStream_t st) {
  if (P.ntiles <= 0) return cudaSuccess;
  k_median<<<P.ntiles, dim3(PS_SIMPLE_BX, PS_SIMPLE_BY), 0, st>>>(P);
  return cudaGetLastError();
}
cudaError_t launch_snapshot(const PsRun& P, float* snap, cudaStream_t st) {
  if (P.ntiles <= 0) return cudaSuccess;
  k_snapshot<<<P.ntiles, dim3(PS_SIMPLE_BX, PS_SIMPLE_BY), 0, st>>>(P, snap);
  return cudaGetLastError();
}
cudaError_t launch_readout(const PsRun& P, float4* out, cudaStream_t st) {
  if (P.ntiles <= 0) return cudaSuccess;
  k_readout<<<P.ntiles, dim3(PS_SIMPLE_BX, PS_SIMPLE_BY), 0, st>>>(P, out);
  return cudaGetLastError();
}
size_t sweep_smem(int wr, int ws) { return eval_smem(wr, ws, true); }

// `tex`: sample sources through their texture objects (tex2Dgather; same bits as the software bilinear).
cudaError_t launch_sweep(const PsRun& P, bool tex, cudaStream_t st) {
  const size_t smem = sweep_smem(P.wr, P.sweep_ws);
  if (P.wr == 6 && P.sweep_ws == 2)
    return tex ? launch(k_sweep<6, 2, true>, P.ntiles, PS_EVAL_NT, smem, st, P)
               : launch(k_sweep<6, 2, false>, P.ntiles, PS_EVAL_NT, smem, st, P);
  if (P.wr == 5 && P.sweep_ws == 2)
    return tex ? launch(k_sweep<5, 2, true>, P.ntiles, PS_EVAL_NT, smem, st, P)
               : launch(k_sweep<5, 2, false>, P.ntiles, PS_EVAL_NT, smem, st, P);
  PsRun Q = P;
  Q.ws = P.sweep_ws;  // the generic kernel reads the window step from the parameters
  return tex ? launch(k_sweep<0, 1, true>, Q.ntiles, PS_EVAL_NT, smem, st, Q)
             : launch(k_sweep<0, 1, false>, Q.ntiles, PS_EVAL_NT, smem, st, Q);
}

// Per-pixel restorer choice of the multi-scale driver (the host driver's `take` rule): the restorer run's plane stays
// where the upsampled plane is invalid (d <= 0) or its evaluated cost exceeds the restorer's by more than `thr`;
// everywhere else the upsampled plane is restored.
__global__ void __launch_bounds__(256) k_restore(const __grid_constant__ PsRun P, const float4* up, const float* cinit,
                                                 float thr) {
  SimpleCtx c;
  if (!simple_px(P, c)) return;
  const long long g = c.it->off + (long long)c.y * c.it->w + c.x;
  const float4 u = up[g];
  const bool take = u.w <= 0.0f || (cinit[g] - P.cost[g]) > thr;
  if (!take) P.plane[g] = u;
}

cudaError_t launch_restore(const PsRun& P, const float4* up, const float* cinit, float thr, cudaStream_t st) {
  if (P.ntiles <= 0) return cudaSuccess;
  k_restore<<<P.ntiles, dim3(PS_SIMPLE_BX, PS_SIMPLE_BY), 0, st>>>(P, up, cinit, thr);
  return cudaGetLastError();
}

// Module constants (propagation offsets); called at session begin, outside any stream capture.
cudaError_t prepare() { return init_constants(); }

cudaError_t launch_rcp_check(int e_lo, int e_hi, unsigned long long* bad, unsigned* first, cudaStream_t st) {
  if (e_lo < -126 || e_hi > 127 || e_lo > e_hi) return cudaErrorInvalidValue;
  k_rcp_check<<<dim3((1u << 23) / 256, e_hi - e_lo + 1), 256, 0, st>>>(e_lo, bad, first);
  return cudaGetLastError();
}

cudaError_t launch_fp32_probe(float* out, int blocks, int iters, cudaStream_t st) {
  k_fp32_probe<<<blocks, 256, 0, st>>>(out, iters, 0.999999f, 1e-7f);
  return cudaGetLastError();
}
cudaError_t launch_setup_lpairs(const PsLevel* lv, const PsPair* pairs, const double* pairs64, const int* has64,
                                PsLPair* out, int nviews, int nlevels, cudaStream_t st) {
  const int n = nviews * nlevels * PS_MAXSRC;
  if (n <= 0) return cudaSuccess;
  k_setup_lpairs<<<(n + 127) / 128, 128, 0, st>>>(lv, pairs, pairs64, has64, out, nviews, nlevels);
  return cudaGetLastError();
}

}  // namespace PS_NS
