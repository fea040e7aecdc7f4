// ps_oracle.cpp — CPU oracle for the PatchStereo hot path.  TEST INFRASTRUCTURE ONLY: it is loaded by tests/,
// by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker; the engine never calls it.
//
// What it restates.  The reference ships no CPU PatchStereo ("This crate has no CPU backend",
// crates/dense/README.md:231-232); its only implementation is the CUDA kernel file
// crates/cuda/src/kernels/patchmatch.cu with the host constants of crates/cuda/src/patchmatch.rs.  This file
// restates that kernel function by function (citations per function), in the reference's own structure: one pixel
// at a time, the reference window read from the image with "0 outside", window weights recomputed per tap, and the
// CPU twins of crates/dense/src/math.rs and crates/dense/src/upsample.rs for the known-answer tests.
//
// Parity pinning.  The reference has no golden PatchStereo outputs (no CPU path, no stored depth maps), so the
// depth-map results are "parity unpinned" against the reference itself.  What IS pinned: the RNG
// (kernel.rs:247-259), FNV-1a (math.rs:31-39), erf / emission / priors / plane transfer (the known answers of
// math.rs:156-213), pyramid levels, intrinsics and the JBU/median plane reproduction (upsample.rs:262-308); see
// tests/test_oracle_kat.py and tests/golden/.
//
// Numerics contract (shared with the engine's parity build).  Compiled with -ffp-contract=off: every operation is a
// correctly rounded binary32 (or binary64) operation in the order written; fused multiply-adds appear only where
// written as fma(); division and square root are IEEE; exp and sincos are the functions of ps_fmath.h.  The places
// where the reference leaves the choice to the compiler (contraction, __expf, rsqrtf, the approximate division of
// its fast-math build, hardware bilinear) are fixed as follows, identically in the engine: the projective
// reciprocal 1/z of the NCC (centre and taps) is the correctly rounded reciprocal (IEEE division); bilinear sample top = fma(ax, p10-p00, p00), bottom likewise, value =
// fma(ay, bot-top, top) on unit-range values (8-bit input: the correctly rounded u/255); tap projection z = fma(H6, sx, fma(H7, sy, H8)) (same for
// the two numerators); window accumulation Ss += w·s, SSs = fma(w·s, s, SSs), IS = fma(w·s, Ik, IS); reference
// statistics S += w·Ik, SS = fma(w·Ik, Ik, SS); every window sum (W, S, SS, Ss, SSs, IS) is kept as two partial
// sums by row parity — even rows and odd rows, each in ascending row and column order — and the total is
// even + odd; rsqrt(a) = 1/sqrt(a); ρ = cov / sqrt(var_r·var_s).
//
// Mode "f64" re-evaluates costs of given hypotheses with every step in binary64 (exp, sqrt, division exact to
// double rounding) and the homography built from FP64 geometry — the FP64 CPU re-evaluation of the precision rule.
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <unordered_map>
#include <vector>

#include "../cumulus3d_b200/csrc/ps_consts.h"
#include "../cumulus3d_b200/csrc/ps_fmath.h"
#include "../include/patchstereo.h"

namespace {

typedef unsigned long long u64;

// ------------------------------------------------------------------------- scalar policy (binary32 / binary64)
inline float fm(float a, float b, float c) { return fmaf(a, b, c); }
inline double fm(double a, double b, double c) { return fma(a, b, c); }
inline float ex(float x) { return ps_expf(x); }
inline double ex(double x) { return exp(x); }
inline float fl(float x) { return floorf(x); }
inline double fl(double x) { return floor(x); }
inline float mn(float a, float b) { return fminf(a, b); }
inline double mn(double a, double b) { return fmin(a, b); }
inline float mx(float a, float b) { return fmaxf(a, b); }
inline double mx(double a, double b) { return fmax(a, b); }
inline float sq(float a) { return sqrtf(a); }
// Tap reciprocal: binary32 is the correctly rounded 1/a (IEEE division; the engine's parity build computes the same
// value with a hardware approximation and one FMA correction); binary64 divides.
inline float rc(float a) { return 1.0f / a; }
inline double rc(double a) { return 1.0 / a; }
inline double sq(double a) { return sqrt(a); }

template <class T>
struct V3 {
  T x, y, z;
};
template <class T>
inline T dot3(V3<T> a, V3<T> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class T>
inline V3<T> cross3(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T>
inline V3<T> nrm3(V3<T> a) {
  T l = (T)1 / sq(mx(dot3(a, a), (T)1e-30f));
  return {a.x * l, a.y * l, a.z * l};
}
struct P4 {
  float x, y, z, w;  // normal, depth
};

// ------------------------------------------------------------------------- RNG (patchmatch.cu:112-125, kernel.rs:247-259)
inline u64 mix64(u64 z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
inline float rnd(u64& s) {
  s += 0x9e3779b97f4a7c15ULL;
  u64 z = mix64(s);
  return ((float)(z >> 40) + 1.0f) * (1.0f / 16777216.0f);
}
inline u64 rng_state(u64 seed, u64 key, int level, int run, int t, int half, u64 pixel) {
  u64 tag = ((u64)level << 48) ^ ((u64)run << 32) ^ ((u64)t << 16) ^ (u64)half;
  return mix64(seed ^ mix64(key ^ mix64(tag)) ^ pixel);
}

// ------------------------------------------------------------------------- scene
struct Img {
  int w = 0, h = 0;
  std::vector<float> px;  // value/255 for u8 input, as is for f32 input
  float fx = 1, fy = 1, cx = 0, cy = 0;
  // RefGlobal::at (patchmatch.cu:139-142): 0 outside.
  float at(int x, int y) const {
    if (x < 0 || y < 0 || x >= w || y >= h) return 0.0f;
    return px[(size_t)y * w + x];
  }
};
struct Pair {
  float r[9], t[3], c[3];
  int src;
  double r64[9], t64[3];
};
struct LPair {
  float A[9], b[3];
  double A64[9], b64[3];
};
struct View {
  u64 key;
  float dmin, dmax;
  std::vector<Img> lv;
  std::vector<Pair> pairs;
  std::vector<LPair> lp;  // [level][src]
};
struct Scene {
  int nl = 0;
  std::vector<View> v;
  ps_pm_params pm;
  ps_filter_params fp;
  u64 seed;
  PsConsts cs;
  int wr, ws, wn;
  const Img& L(int view, int level) const { return v[view].lv[level]; }
};

// A = K_j R K^-1, b = K_j t in binary64 (crates/cuda/src/patchmatch.rs:132-151), then rounded to binary32.
void level_pair(const float* kr, const float* kj, const double* r, const double* t, LPair& o) {
  const double fx = kr[0], fy = kr[1], cx = kr[2], cy = kr[3];
  const double kinv[3][3] = {{1.0 / fx, 0.0, -cx / fx}, {0.0, 1.0 / fy, -cy / fy}, {0.0, 0.0, 1.0}};
  const double km[3][3] = {{(double)kj[0], 0.0, (double)kj[2]}, {0.0, (double)kj[1], (double)kj[3]}, {0.0, 0.0, 1.0}};
  double krm[3][3];
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) krm[i][k] = km[i][0] * r[0 * 3 + k] + km[i][1] * r[1 * 3 + k] + km[i][2] * r[2 * 3 + k];
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) {
      o.A64[i * 3 + k] = krm[i][0] * kinv[0][k] + krm[i][1] * kinv[1][k] + krm[i][2] * kinv[2][k];
      o.A[i * 3 + k] = (float)o.A64[i * 3 + k];
    }
  for (int i = 0; i < 3; ++i) {
    o.b64[i] = km[i][0] * t[0] + km[i][1] * t[1] + km[i][2] * t[2];
    o.b[i] = (float)o.b64[i];
  }
}

bool load_scene(const ps_kernel_input* in, Scene& sc) {
  if (!in || in->num_levels < 1) return false;
  sc.nl = (int)in->num_levels;
  sc.pm = in->pm;
  sc.fp = in->filter;
  sc.seed = in->seed;
  sc.cs = ps_session_consts(&sc.pm, &sc.fp);
  sc.wr = sc.pm.window_radius;
  sc.ws = sc.pm.window_step;
  sc.wn = (2 * sc.wr) / sc.ws + 1;
  sc.v.resize(in->num_views);
  for (uint32_t i = 0; i < in->num_views; ++i) {
    const ps_kernel_view& kv = in->views[i];
    View& v = sc.v[i];
    v.key = kv.key;
    v.dmin = kv.depth_min;
    v.dmax = kv.depth_max;
    v.lv.resize(sc.nl);
    for (int l = 0; l < sc.nl; ++l) {
      const ps_level_image& li = kv.levels[l];
      Img& im = v.lv[l];
      im.w = (int)li.width;
      im.h = (int)li.height;
      im.fx = li.k[0];
      im.fy = li.k[1];
      im.cx = li.k[2];
      im.cy = li.k[3];
      im.px.resize((size_t)im.w * im.h);
      const size_t stride = li.stride ? li.stride : li.width;
      for (int y = 0; y < im.h; ++y)
        for (int x = 0; x < im.w; ++x)
          im.px[(size_t)y * im.w + x] = li.format == PS_IMAGE_U8
                                            ? ps_u8_unit(((const uint8_t*)li.pixels)[y * stride + x])
                                            : ((const float*)li.pixels)[y * stride + x];
    }
    v.pairs.resize(kv.num_sources);
    for (uint32_t j = 0; j < kv.num_sources; ++j) {
      Pair& p = v.pairs[j];
      memcpy(p.r, kv.pairs[j].r, sizeof p.r);
      memcpy(p.t, kv.pairs[j].t, sizeof p.t);
      memcpy(p.c, kv.pairs[j].center, sizeof p.c);
      p.src = (int)kv.sources[j];
      for (int k = 0; k < 9; ++k) p.r64[k] = kv.pairs_f64 ? kv.pairs_f64[j * 15 + k] : (double)p.r[k];
      for (int k = 0; k < 3; ++k) p.t64[k] = kv.pairs_f64 ? kv.pairs_f64[j * 15 + 9 + k] : (double)p.t[k];
    }
  }
  for (uint32_t i = 0; i < in->num_views; ++i) {
    View& v = sc.v[i];
    v.lp.resize((size_t)sc.nl * v.pairs.size());
    for (int l = 0; l < sc.nl; ++l)
      for (size_t j = 0; j < v.pairs.size(); ++j) {
        const ps_level_image& a = in->views[i].levels[l];
        const ps_level_image& b = in->views[v.pairs[j].src].levels[l];
        level_pair(a.k, b.k, v.pairs[j].r64, v.pairs[j].t64, v.lp[l * v.pairs.size() + j]);
      }
  }
  return true;
}

// ------------------------------------------------------------------------- per-pixel restatement
struct Run {
  const Scene* sc;
  int view, level;
  int geometric, run_id, t, color, topk, use_prior;
  float tau_good, eps, phi;
  const std::vector<std::vector<float>>* snap;  // per view (empty = absent)
  const float* proposal = nullptr;  // learned init: 4 floats per pixel, d > 0 replaces the random draw
};

template <class T>
struct RS {
  T ic, W, mu, var;
};

// Source sample, integer-centre convention, 0 outside (patchmatch.cu:169-192, software path).
template <class T>
T sample(const Img& S, T u, T v) {
  T xf = fl(u), yf = fl(v);
  T ax = u - xf, ay = v - yf;
  // integer footprint; the clamp only guards the conversion and keeps out-of-image footprints out of the image
  const int x0 = (int)mn(mx(xf, (T)-2), (T)S.w), y0 = (int)mn(mx(yf, (T)-2), (T)S.h);
  T p00 = (T)S.at(x0, y0), p10 = (T)S.at(x0 + 1, y0), p01 = (T)S.at(x0, y0 + 1), p11 = (T)S.at(x0 + 1, y0 + 1);
  T top = fm(ax, p10 - p00, p00);
  T bot = fm(ax, p11 - p01, p01);
  return fm(ay, bot - top, top);
}

// ref_stats (patchmatch.cu:199-223), window sums split by row parity (even rows and odd rows accumulate
// separately in ascending row order; total = even + odd).
template <class T>
RS<T> ref_stats(const Scene& sc, const Img& R, int x, int y) {
  RS<T> s;
  s.ic = (T)R.at(x, y);
  T W[2] = {0, 0}, S[2] = {0, 0}, SS[2] = {0, 0};
  const T inv2s = (T)sc.cs.inv2s, inv2c = (T)sc.cs.inv2c;
  for (int a = 0; a < sc.wn; ++a) {
    int dy = -sc.wr + a * sc.ws;
    const int p = a & 1;
    for (int b = 0; b < sc.wn; ++b) {
      int dx = -sc.wr + b * sc.ws;
      T ik = (T)R.at(x + dx, y + dy);
      T d = s.ic - ik;
      T w = ex(-(T)(dx * dx + dy * dy) * inv2s - d * d * inv2c);
      T wi = w * ik;
      W[p] = W[p] + w;
      S[p] = S[p] + wi;
      SS[p] = fm(wi, ik, SS[p]);
    }
  }
  s.W = W[0] + W[1];
  const T St = S[0] + S[1], SSt = SS[0] + SS[1];
  s.mu = St / s.W;
  s.var = SSt / s.W - s.mu * s.mu;
  return s;
}

// Homography (patchmatch.cu:225-242).
template <class T>
bool homography(const Img& R, const LPair& L, T x, T y, const P4& h, T* H) {
  T ifx = (T)1 / (T)R.fx, ify = (T)1 / (T)R.fy;
  V3<T> n = {(T)h.x, (T)h.y, (T)h.z};
  V3<T> ray = {(x - (T)R.cx) * ifx, (y - (T)R.cy) * ify, (T)1};
  T delta = (T)h.w * dot3(n, ray);
  if (!(delta < (T)-1e-12f)) return false;
  T id = (T)1 / delta;
  T u0 = n.x * ifx, u1 = n.y * ify;
  T u2 = n.z - u0 * (T)R.cx - u1 * (T)R.cy;
  const bool d64 = sizeof(T) == 8;
  for (int r = 0; r < 3; ++r) {
    T br = (d64 ? (T)L.b64[r] : (T)L.b[r]) * id;
    H[r * 3 + 0] = (d64 ? (T)L.A64[r * 3 + 0] : (T)L.A[r * 3 + 0]) + br * u0;
    H[r * 3 + 1] = (d64 ? (T)L.A64[r * 3 + 1] : (T)L.A[r * 3 + 1]) + br * u1;
    H[r * 3 + 2] = (d64 ? (T)L.A64[r * 3 + 2] : (T)L.A[r * 3 + 2]) + br * u2;
  }
  return true;
}

// NCC cost (patchmatch.cu:245-290), weights recomputed per tap as the reference's global-memory path does.
template <class T>
T ncc_cost(const Scene& sc, const Img& R, const RS<T>& rs, const Img& S, const T* H, int x, int y) {
  T fx = (T)x, fy = (T)y;
  T z = fm(H[6], fx, fm(H[7], fy, H[8]));
  if (!(z > (T)1e-8f)) return 2;
  T iz = rc(z);
  T u = fm(H[0], fx, fm(H[1], fy, H[2])) * iz, v = fm(H[3], fx, fm(H[4], fy, H[5])) * iz;
  if (!(u >= 0 && v >= 0 && u <= (T)S.w - (T)1 && v <= (T)S.h - (T)1)) return 2;
  if (rs.var < (T)1e-5f) return 2;
  const T inv2s = (T)sc.cs.inv2s, inv2c = (T)sc.cs.inv2c;
  T Ss[2] = {0, 0}, SSs[2] = {0, 0}, IS[2] = {0, 0};
  for (int a = 0; a < sc.wn; ++a) {
    int dy = -sc.wr + a * sc.ws;
    const int p = a & 1;
    T sy = fy + (T)dy;
    for (int b = 0; b < sc.wn; ++b) {
      int dx = -sc.wr + b * sc.ws;
      T sx = fx + (T)dx;
      T ik = (T)R.at(x + dx, y + dy);
      T d = rs.ic - ik;
      T w = ex(-(T)(dx * dx + dy * dy) * inv2s - d * d * inv2c);
      T zz = fm(H[6], sx, fm(H[7], sy, H[8]));
      T sv = 0;
      if (zz > (T)1e-8f) {
        T izz = rc(zz);
        sv = sample<T>(S, fm(H[0], sx, fm(H[1], sy, H[2])) * izz, fm(H[3], sx, fm(H[4], sy, H[5])) * izz);
      }
      T wsv = w * sv;
      Ss[p] = Ss[p] + wsv;
      SSs[p] = fm(wsv, sv, SSs[p]);
      IS[p] = fm(wsv, ik, IS[p]);
    }
  }
  const T Sst = Ss[0] + Ss[1], SSst = SSs[0] + SSs[1], ISt = IS[0] + IS[1];
  T iW = (T)1 / rs.W;
  T mus = Sst * iW;
  T vars = SSst * iW - mus * mus;
  if (vars < (T)1e-5f) return 2;
  T cov = ISt * iW - rs.mu * mus;
  T c = (T)1 - cov / sq(rs.var * vars);
  return mn(mx(c, (T)0), (T)2);
}

// Forward/backward reprojection error (patchmatch.cu:292-314).
const float INF_ERR = 1e30f;
template <class T>
T geo_error(const Run& r, const Img& R, const Img& S, const Pair& pr, int x, int y, T d) {
  const std::vector<float>& sm = (*r.snap)[pr.src];
  if (sm.empty()) return (T)INF_ERR;
  const bool d64 = sizeof(T) == 8;
  auto rr = [&](int k) { return d64 ? (T)pr.r64[k] : (T)pr.r[k]; };
  auto tt = [&](int k) { return d64 ? (T)pr.t64[k] : (T)pr.t[k]; };
  V3<T> X = {((T)x - (T)R.cx) / (T)R.fx * d, ((T)y - (T)R.cy) / (T)R.fy * d, d};
  T xj = rr(0) * X.x + rr(1) * X.y + rr(2) * X.z + tt(0);
  T yj = rr(3) * X.x + rr(4) * X.y + rr(5) * X.z + tt(1);
  T zj = rr(6) * X.x + rr(7) * X.y + rr(8) * X.z + tt(2);
  if (!(zj > (T)1e-8f)) return (T)INF_ERR;
  T u = (T)S.fx * xj / zj + (T)S.cx, v = (T)S.fy * yj / zj + (T)S.cy;
  T uf = fl(u + (T)0.5f), vf = fl(v + (T)0.5f);
  if (!(uf >= 0 && vf >= 0 && uf < (T)S.w && vf < (T)S.h)) return (T)INF_ERR;
  T dj = (T)sm[(size_t)vf * S.w + (size_t)uf];
  if (!(dj > 0)) return (T)INF_ERR;
  V3<T> Yj = {(u - (T)S.cx) / (T)S.fx * dj, (v - (T)S.cy) / (T)S.fy * dj, dj};
  V3<T> q = {Yj.x - tt(0), Yj.y - tt(1), Yj.z - tt(2)};
  T Yx = rr(0) * q.x + rr(3) * q.y + rr(6) * q.z;
  T Yy = rr(1) * q.x + rr(4) * q.y + rr(7) * q.z;
  T Yz = rr(2) * q.x + rr(5) * q.y + rr(8) * q.z;
  if (!(Yz > (T)1e-8f)) return (T)INF_ERR;
  T cx = (T)R.fx * Yx / Yz + (T)R.cx - (T)x, cy = (T)R.fy * Yy / Yz + (T)R.cy - (T)y;
  return sq(cx * cx + cy * cy);
}

template <class T>
T pair_cost(const Run& r, const Img& R, const RS<T>& rs, int j, int x, int y, const P4& h, T* geo) {
  const Scene& sc = *r.sc;
  const View& vw = sc.v[r.view];
  const Pair& pr = vw.pairs[j];
  const Img& S = sc.L(pr.src, r.level);
  const LPair& lp = vw.lp[(size_t)r.level * vw.pairs.size() + j];
  T H[9];
  T c = 2;
  if (homography<T>(R, lp, (T)x, (T)y, h, H)) c = ncc_cost<T>(sc, R, rs, S, H, x, y);
  if (r.geometric) *geo = mn(geo_error<T>(r, R, S, pr, x, y, (T)h.w), (T)sc.cs.gmax);
  return c;
}

// topk_cost (patchmatch.cu:327-345).
template <class T>
T topk_cost(const Run& r, const Img& R, const RS<T>& rs, int x, int y, const P4& h) {
  const View& vw = r.sc->v[r.view];
  T b0 = (T)1e30f, b1 = (T)1e30f, b2 = (T)1e30f;
  const int nsrc = (int)vw.pairs.size();
  for (int j = 0; j < nsrc; ++j) {
    T g = 0;
    T c = pair_cost<T>(r, R, rs, j, x, y, h, &g);
    if (r.geometric) c += (T)r.sc->cs.lambda * g;
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
  int k = std::min(r.topk, nsrc);
  T s = b0;
  if (k >= 2) s += b1;
  if (k >= 3) s += b2;
  return k > 0 ? s / (T)k : (T)2;
}

V3<float> pixel_ray(const Img& R, int x, int y) { return {((float)x - R.cx) / R.fx, ((float)y - R.cy) / R.fy, 1.0f}; }

// random_normal / random_depth / perturb_normal (patchmatch.cu:348-384).
V3<float> random_normal(u64& st, V3<float> ray) {
  V3<float> n = {0.f, 0.f, -1.f};
  for (int k = 0; k < 64; ++k) {
    float v1 = 2.f * rnd(st) - 1.f, v2 = 2.f * rnd(st) - 1.f;
    float s = v1 * v1 + v2 * v2;
    if (s < 1.f && s > 0.f) {
      float r = 2.f * sqrtf(1.f - s);
      n = {v1 * r, v2 * r, 1.f - 2.f * s};
      break;
    }
  }
  if (dot3(n, ray) > 0.f) n = {-n.x, -n.y, -n.z};
  return n;
}
float random_depth(u64& st, float dmin, float dmax) {
  float a = 1.f / dmax, b = 1.f / dmin;
  return 1.f / (a + rnd(st) * (b - a));
}
V3<float> perturb_normal(u64& st, V3<float> n, V3<float> ray, float phi) {
  V3<float> a = random_normal(st, {0.f, 0.f, 0.f});
  V3<float> ax = cross3(a, n);
  float l2 = dot3(ax, ax);
  float ang = rnd(st) * phi;
  if (l2 < 1e-12f) return n;
  ax = nrm3(ax);
  V3<float> bn = cross3(ax, n);
  for (int k = 0; k < 4; ++k) {
    float sa, ca;
    ps_sincosf(ang, &sa, &ca);
    V3<float> m = {n.x * ca + bn.x * sa, n.y * ca + bn.y * sa, n.z * ca + bn.z * sa};
    if (dot3(m, ray) < 0.f) return nrm3(m);
    ang *= 0.5f;
  }
  return n;
}

// view_prior (patchmatch.cu:388-422).
float view_prior(const Scene& sc, const Img& R, const Pair& pr, const float* H, bool hok, int x, int y, const P4& h) {
  if (!hok) return 0.f;
  V3<float> ray = pixel_ray(R, x, y);
  V3<float> X = {ray.x * h.w, ray.y * h.w, h.w};
  V3<float> S = {pr.c[0] - X.x, pr.c[1] - X.y, pr.c[2] - X.z};
  float ls = sqrtf(dot3(S, S)), lx = sqrtf(dot3(X, X));
  if (ls <= 0.f || lx <= 0.f) return 0.f;
  float cost = -dot3(S, X) / (ls * lx);
  float tri = 1.f;
  if (cost > sc.cs.cos_tri_min) {
    float s = 1.f - (1.f - cost) / (1.f - sc.cs.cos_tri_min);
    tri = fminf(fmaxf(1.f - s * s, 0.f), 1.f);
  }
  float cphi = dot3(S, V3<float>{h.x, h.y, h.z}) / ls;
  float xi = 1.f - fmaxf(0.f, cphi);
  float inc = ps_expf(-xi * xi * sc.cs.inv2inc);
  float r = (float)sc.wr;
  float cxs[4] = {x - r, x - r, x + r, x + r};
  float cys[4] = {y - r, y + r, y + r, y - r};
  float px[4], py[4];
  for (int k = 0; k < 4; ++k) {
    float z = H[6] * cxs[k] + H[7] * cys[k] + H[8];
    if (!(z > 1e-8f)) return 0.f;
    px[k] = (H[0] * cxs[k] + H[1] * cys[k] + H[2]) / z;
    py[k] = (H[3] * cxs[k] + H[4] * cys[k] + H[5]) / z;
  }
  float area = 0.f;
  for (int k = 0; k < 4; ++k) area += px[k] * py[(k + 1) & 3] - px[(k + 1) & 3] * py[k];
  area = 0.5f * fabsf(area);
  float aref = (2.f * r + 1.f) * (2.f * r + 1.f);
  if (!(area > 0.f)) return 0.f;
  float res = fminf(area / aref, aref / area);
  return tri * inc * res;
}

// Region offsets for the "up" direction (patchmatch.cu:425) and the 90° rotation (:427-436).
const int V_OFF[7][2] = {{0, -1}, {-1, -2}, {1, -2}, {-2, -3}, {2, -3}, {-3, -4}, {3, -4}};
void rot_dir(int dir, int dx, int dy, int& ox, int& oy) {
  ox = dx;
  oy = dy;
  for (int k = 0; k < dir; ++k) {
    int t = ox;
    ox = -oy;
    oy = t;
  }
}

struct State {
  int w, h;
  std::vector<P4> plane;
  std::vector<float> cost;
  std::vector<uint8_t> bview;
  std::vector<P4> prior;
};

// One red-black half step of one pixel (patchmatch.cu:439-657).  Reads opposite-colour neighbours only.
void half_pixel(const Run& r, State& st, int x, int y) {
  const Scene& sc = *r.sc;
  const View& vd = sc.v[r.view];
  const Img& R = sc.L(r.view, r.level);
  const int w = st.w, h = st.h;
  const int pix = y * w + x;
  const V3<float> ray = pixel_ray(R, x, y);
  P4 hyp[9];
  hyp[0] = st.plane[pix];
  for (int rg = 0; rg < 8; ++rg) {
    int dir = rg & 3;
    bool strip = rg >= 4;
    int cnt = strip ? 11 : 7;
    float best = 1e30f;
    int bq = -1, bx = 0, by = 0;
    for (int k = 0; k < cnt; ++k) {
      int dx, dy;
      if (strip) rot_dir(dir, 0, -(3 + 2 * k), dx, dy);
      else rot_dir(dir, V_OFF[k][0], V_OFF[k][1], dx, dy);
      int qx = x + dx, qy = y + dy;
      if (qx < 0 || qy < 0 || qx >= w || qy >= h) continue;
      float c = st.cost[qy * w + qx];
      if (c < best) {
        best = c;
        bq = qy * w + qx;
        bx = qx;
        by = qy;
      }
    }
    hyp[1 + rg] = hyp[0];
    if (bq >= 0) {
      P4 q = st.plane[bq];
      V3<float> n = {q.x, q.y, q.z};
      V3<float> rq = pixel_ray(R, bx, by);
      float den = dot3(n, ray);
      if (den < -1e-6f && q.w > 0.f) {
        float d = q.w * dot3(n, rq) / den;
        if (d > 0.f && std::isfinite(d)) hyp[1 + rg] = {n.x, n.y, n.z, d};
      }
    }
  }
  const RS<float> rs = ref_stats<float>(sc, R, x, y);
  const int vprev = st.bview[pix];
  const int nsrc = (int)vd.pairs.size();
  float num[9] = {0}, numf[9] = {0};
  float den = 0.f, wbest = 0.f, denf = 0.f;
  int vbest = 255;
  float wv[PS_MAX_SOURCES];
  for (int j = 0; j < nsrc; ++j) {
    const Pair& pr = vd.pairs[j];
    const Img& S = sc.L(pr.src, r.level);
    const LPair& lp = vd.lp[(size_t)r.level * nsrc + j];
    float m[9], gg[9];
    float prior;
    {
      float H[9];
      bool ok = homography<float>(R, lp, (float)x, (float)y, hyp[0], H);
      prior = view_prior(sc, R, pr, H, ok, x, y, hyp[0]);
      wv[j] = 0.f;
      if (!(prior > 0.f)) continue;
      m[0] = ok ? ncc_cost<float>(sc, R, rs, S, H, x, y) : 2.f;
      gg[0] = r.geometric ? fminf(geo_error<float>(r, R, S, pr, x, y, hyp[0].w), sc.cs.gmax) : 0.f;
    }
    for (int i = 1; i < 9; ++i) {
      float H[9];
      bool ok = homography<float>(R, lp, (float)x, (float)y, hyp[i], H);
      m[i] = ok ? ncc_cost<float>(sc, R, rs, S, H, x, y) : 2.f;
      gg[i] = r.geometric ? fminf(geo_error<float>(r, R, S, pr, x, y, hyp[i].w), sc.cs.gmax) : 0.f;
    }
    int good = 0, bad = 0;
    float conf = 0.f;
    for (int i = 1; i < 9; ++i) {
      if (m[i] < r.tau_good) {
        good++;
        conf += ps_expf(-m[i] * m[i] * sc.cs.inv2beta2);
      }
      if (m[i] > sc.cs.tau_bad) bad++;
    }
    bool adopt = good > sc.cs.n1 && bad < sc.cs.n2;
    bool isprev = j == vprev;
    float wp = adopt ? (isprev ? 2.f : 1.f) * conf / (float)good : (isprev ? sc.cs.prev_w : 0.f);
    float w2 = wp * prior;
    wv[j] = w2 > 0.f ? w2 : -prior;
    for (int i = 0; i < 9; ++i) numf[i] += prior * (m[i] + sc.cs.lambda * gg[i]);
    denf += prior;
    if (w2 > 0.f) {
      for (int i = 0; i < 9; ++i) num[i] += w2 * (m[i] + sc.cs.lambda * gg[i]);
      den += w2;
      if (w2 > wbest) {
        wbest = w2;
        vbest = j;
      }
    }
  }
  float agg[9];
  int bi9 = 0;
  if (den > 0.f) {
    for (int i = 0; i < 9; ++i) agg[i] = num[i] / den;
    for (int i = 1; i < 9; ++i)
      if (agg[i] < agg[bi9]) bi9 = i;
  } else if (denf > 0.f) {
    for (int i = 0; i < 9; ++i) agg[i] = numf[i] / denf;
    for (int i = 1; i < 9; ++i)
      if (agg[i] < agg[bi9]) bi9 = i;
    for (int j = 0; j < nsrc; ++j) wv[j] = -wv[j];
    den = denf;
  } else {
    for (int i = 0; i < 9; ++i) agg[i] = 2.f;
  }
  P4 best = hyp[bi9];
  float bcost = agg[bi9];
  u64 s = rng_state(sc.seed, vd.key, r.level, r.run_id, r.t, r.color, (u64)pix);
  float d_r = random_depth(s, vd.dmin, vd.dmax);
  V3<float> n_r = random_normal(s, ray);
  float u = 2.f * rnd(s) - 1.f;
  float inv = best.w > 0.f ? (1.f / best.w) * (1.f + u * r.eps) : -1.f;
  float d_p = inv > 0.f ? 1.f / inv : d_r;
  if (!(best.w > 0.f)) best.w = d_r;
  V3<float> n0 = {best.x, best.y, best.z};
  V3<float> n_p = perturb_normal(s, n0, ray, r.phi);
  P4 cand[6] = {{n0.x, n0.y, n0.z, d_r},        {n_r.x, n_r.y, n_r.z, best.w}, {n_r.x, n_r.y, n_r.z, d_r},
                {n0.x, n0.y, n0.z, d_p},        {n_p.x, n_p.y, n_p.z, best.w}, {n_p.x, n_p.y, n_p.z, d_p}};
  auto weighted = [&](const P4& c) {
    if (!(den > 0.f)) return 2.f;
    float nm = 0.f;
    for (int j = 0; j < nsrc; ++j) {
      if (!(wv[j] > 0.f)) continue;
      float g = 0.f;
      float mm = pair_cost<float>(r, R, rs, j, x, y, c, &g);
      nm += wv[j] * (mm + sc.cs.lambda * g);
    }
    return nm / den;
  };
  for (int c = 0; c < 6; ++c) {
    float cc = weighted(cand[c]);
    if (cc < bcost) {
      bcost = cc;
      best = cand[c];
    }
  }
  if (r.use_prior && rs.var < sc.cs.weak_var) {
    P4 q = st.prior[pix];
    if (q.w > 0.f && dot3(V3<float>{q.x, q.y, q.z}, ray) < 0.f) {
      float cc = weighted(q);
      if (cc < bcost) {
        bcost = cc;
        best = q;
      }
    }
  }
  st.plane[pix] = best;
  st.cost[pix] = bcost;
  st.bview[pix] = (uint8_t)vbest;
}

// pm_eval (patchmatch.cu:661-692).
void eval_pixel(const Run& r, State& st, int x, int y, int mode, int random_init) {
  const Scene& sc = *r.sc;
  const View& vd = sc.v[r.view];
  const Img& R = sc.L(r.view, r.level);
  const int pix = y * st.w + x;
  V3<float> ray = pixel_ray(R, x, y);
  P4 h = st.plane[pix];
  if (mode == 1 && random_init) {
    u64 s = rng_state(sc.seed, vd.key, r.level, r.run_id, 0xFFFF, 0, (u64)pix);
    float d = random_depth(s, vd.dmin, vd.dmax);
    V3<float> n = random_normal(s, ray);
    h = {n.x, n.y, n.z, d};
    if (r.proposal && r.proposal[4 * pix + 3] > 0.f) {
      const float* q = r.proposal + 4 * pix;
      h = {q[0], q[1], q[2], q[3]};
    }
    st.plane[pix] = h;
  }
  float c = 2.f;
  if (h.w > 0.f) {
    RS<float> rs = ref_stats<float>(sc, R, x, y);
    c = topk_cost<float>(r, R, rs, x, y, h);
  }
  st.cost[pix] = c;
  if (mode == 1) st.bview[pix] = 255;
}

// pm_filter (patchmatch.cu:695-737).
int filter_pixel(const Run& r, const State& st, int x, int y) {
  const Scene& sc = *r.sc;
  const View& vd = sc.v[r.view];
  const Img& R = sc.L(r.view, r.level);
  const int pix = y * st.w + x;
  P4 h = st.plane[pix];
  int count = 0;
  if (h.w > 0.f) {
    RS<float> rs = ref_stats<float>(sc, R, x, y);
    V3<float> ray = pixel_ray(R, x, y);
    V3<float> X = {ray.x * h.w, ray.y * h.w, h.w};
    float lx = sqrtf(dot3(X, X));
    const int nsrc = (int)vd.pairs.size();
    for (int j = 0; j < nsrc; ++j) {
      const Pair& pr = vd.pairs[j];
      const Img& S = sc.L(pr.src, r.level);
      V3<float> Sv = {pr.c[0] - X.x, pr.c[1] - X.y, pr.c[2] - X.z};
      float ls = sqrtf(dot3(Sv, Sv));
      if (!(ls > 0.f)) continue;
      float cost = -dot3(Sv, X) / (ls * lx);
      if (cost > sc.cs.cos_filter_tri) continue;
      float cphi = dot3(Sv, V3<float>{h.x, h.y, h.z}) / ls;
      if (cphi <= 0.f) continue;
      float H[9];
      if (!homography<float>(R, vd.lp[(size_t)r.level * nsrc + j], (float)x, (float)y, h, H)) continue;
      float m = ncc_cost<float>(sc, R, rs, S, H, x, y);
      float e = sc.cs.ncc_norm * ps_expf(-m * m * sc.cs.inv2ncc);
      if (e / (e + 0.5f) < sc.cs.q_min) continue;
      if (geo_error<float>(r, R, S, pr, x, y, h.w) > sc.cs.filter_gmax) continue;
      count++;
    }
  }
  return std::min(count, 255);
}

void to_state(const ps_view_state& vs, State& st, bool planes) {
  st.w = (int)vs.width;
  st.h = (int)vs.height;
  const size_t n = (size_t)st.w * st.h;
  st.plane.assign(n, P4{0, 0, 0, 0});
  st.cost.assign(n, 2.0f);
  st.bview.assign(n, 255);
  if (planes)
    for (size_t p = 0; p < n; ++p) st.plane[p] = {vs.normal[3 * p], vs.normal[3 * p + 1], vs.normal[3 * p + 2], vs.depth[p]};
  if (vs.prior) {
    st.prior.resize(n);
    memcpy(st.prior.data(), vs.prior, n * sizeof(P4));
  }
}
void from_state(const State& st, ps_view_state& vs) {
  const size_t n = (size_t)st.w * st.h;
  for (size_t p = 0; p < n; ++p) {
    vs.normal[3 * p] = st.plane[p].x;
    vs.normal[3 * p + 1] = st.plane[p].y;
    vs.normal[3 * p + 2] = st.plane[p].z;
    vs.depth[p] = st.plane[p].w;
    vs.cost[p] = st.cost[p];
  }
}

std::vector<std::vector<float>> snapshot_maps(const Scene& sc, const ps_depth_snapshot* snap) {
  std::vector<std::vector<float>> m(sc.v.size());
  if (!snap) return m;
  for (size_t v = 0; v < sc.v.size(); ++v)
    if (v < snap->num_maps && snap->maps && snap->maps[v]) {
      const Img& L = sc.L((int)v, (int)snap->level);
      // a map of another size is left out (crates/cuda/src/patchmatch.rs:573-604)
      if (snap->map_lengths && snap->map_lengths[v] != (uint64_t)L.w * L.h) continue;
      m[v].assign(snap->maps[v], snap->maps[v] + (size_t)L.w * L.h);
    }
  return m;
}

int set_threads(int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  return 0;
}

}  // namespace

// ================================================================================================ C entry points
extern "C" {

// PatchMatchSession::run restated (crates/cuda/src/patchmatch.rs:752-799): per view, run start (evaluate mode 1)
// then `iterations` × (colour 0, colour 1) half steps.
// Rows [y0, y1) only (y1 <= 0: all rows): the timing sample of the CPU baseline runs a band of rows, whose cost is
// proportional to its pixel count; parity tests always run every row.
int oracle_run_init(const ps_kernel_input* in, const uint32_t* views, size_t n, ps_view_state* states,
                    const ps_run_params* p, const ps_depth_snapshot* snap, const float* const* proposals, int threads,
                    int y0, int y1) {
  Scene sc;
  if (!load_scene(in, sc) || !p) return PS_EINVAL;
  if (p->geometric && !snap) return PS_EINVAL;
  set_threads(threads);
  std::vector<std::vector<float>> maps = snapshot_maps(sc, snap);
  for (size_t i = 0; i < n; ++i) {
    State st;
    to_state(states[i], st, !p->random_init);
    Run r;
    r.sc = &sc;
    r.view = (int)views[i];
    r.level = (int)p->level;
    r.geometric = p->geometric;
    r.run_id = (int)p->run_id;
    r.topk = sc.cs.topk;
    r.use_prior = p->use_prior && states[i].prior ? 1 : 0;
    r.snap = &maps;
    r.t = 0;
    r.color = 0;
    r.tau_good = r.eps = r.phi = 0;
    r.proposal = (p->random_init == PS_INIT_PROPOSAL && proposals) ? proposals[i] : nullptr;
    // work items of CHUNK columns of one row (pixels of one colour are independent, so the split changes no bits;
    // small items keep the threads balanced on a narrow band)
    constexpr int CHUNK = 64;
    const int ya = std::max(y0, 0), yb = y1 > 0 ? std::min(y1, st.h) : st.h;
    const int cx = (st.w + CHUNK - 1) / CHUNK;
    const long long items = (long long)std::max(yb - ya, 0) * cx;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long k = 0; k < items; ++k) {
      const int y = ya + (int)(k / cx), xa = (int)(k % cx) * CHUNK, xb = std::min(xa + CHUNK, st.w);
      for (int x = xa; x < xb; ++x) eval_pixel(r, st, x, y, 1, p->random_init);
    }
    for (uint32_t t = 0; t < p->iterations; ++t) {
      r.t = (int)t;
      ps_iter_consts(&sc.pm, p->geometric, (int)t, &r.tau_good, &r.eps, &r.phi);
      for (int color = 0; color < 2; ++color) {
        r.color = color;
#pragma omp parallel for schedule(dynamic, 1)
        for (long long k = 0; k < items; ++k) {
          const int y = ya + (int)(k / cx), xa = (int)(k % cx) * CHUNK, xb = std::min(xa + CHUNK, st.w);
          for (int x = xa + ((y + color) & 1); x < xb; x += 2) half_pixel(r, st, x, y);
        }
      }
    }
    from_state(st, states[i]);
  }
  return PS_OK;
}

int oracle_run_rows(const ps_kernel_input* in, const uint32_t* views, size_t n, ps_view_state* states,
                    const ps_run_params* p, const ps_depth_snapshot* snap, int threads, int y0, int y1) {
  return oracle_run_init(in, views, n, states, p, snap, nullptr, threads, y0, y1);
}

int oracle_run(const ps_kernel_input* in, const uint32_t* views, size_t n, ps_view_state* states,
               const ps_run_params* p, const ps_depth_snapshot* snap, int threads) {
  return oracle_run_rows(in, views, n, states, p, snap, threads, 0, 0);
}

// Plane-sweep network input of one view (the engine's ps_sweep_volume; no reference counterpart): per pixel, bf16
// bits of [image, 32 costs, 15 zeros] where cost k is the mean over the first min(2, nsrc) sources of the NCC cost of
// the plane (n, 1/i_k) at the pixel, n = `normal` (NULL: fronto-parallel (0, 0, -1)),
// i_k = fma((2k+1)/64, 1/dmin - 1/dmax, 1/dmax), window radius as the session's and step 2 (2 where the homography
// fails).  Rows of `row_pixels` pixels.
int oracle_sweep(const ps_kernel_input* in, uint32_t level, uint32_t view, uint16_t* out, uint32_t row_pixels,
                 const float* normal, int threads) {
  Scene sc;
  if (!load_scene(in, sc) || view >= sc.v.size() || (int)level >= sc.nl || !out) return PS_EINVAL;
  sc.ws = 2;
  sc.wn = (2 * sc.wr) / sc.ws + 1;
  set_threads(threads);
  const View& vd = sc.v[view];
  const Img& R = sc.L((int)view, (int)level);
  if ((int)row_pixels < R.w) return PS_EINVAL;
  const int nsrc = (int)vd.pairs.size(), nuse = std::min(nsrc, 2);
  const float inear = 1.0f / vd.dmin, ifar = 1.0f / vd.dmax;
  auto bf16 = [](float v) -> uint16_t {  // round to nearest even (finite values)
    uint32_t u;
    memcpy(&u, &v, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
  };
#pragma omp parallel for schedule(dynamic, 1)
  for (int y = 0; y < R.h; ++y)
    for (int x = 0; x < R.w; ++x) {
      uint16_t* o = out + ((size_t)y * row_pixels + x) * PS_NET_CH_IN;
      const RS<float> rs = ref_stats<float>(sc, R, x, y);
      o[0] = bf16(R.at(x, y));
      for (int k = 0; k < PS_SWEEP_PLANES; ++k) {
        const float id = std::fma((float)(2 * k + 1) * (1.0f / 64.0f), inear - ifar, ifar);
        const P4 h = {normal ? normal[0] : 0.0f, normal ? normal[1] : 0.0f, normal ? normal[2] : -1.0f, 1.0f / id};
        float c = 0.0f;
        for (int j = 0; j < nuse; ++j) {
          const Img& S = sc.L(vd.pairs[j].src, (int)level);
          float H[9];
          c += homography<float>(R, vd.lp[(size_t)level * nsrc + j], (float)x, (float)y, h, H)
                   ? ncc_cost<float>(sc, R, rs, S, H, x, y)
                   : 2.0f;
        }
        c = nuse == 2 ? c * 0.5f : (nuse == 1 ? c : 2.0f);
        o[1 + k] = bf16(c);
      }
      for (int k = 1 + PS_SWEEP_PLANES; k < PS_NET_CH_IN; ++k) o[k] = 0;
    }
  return PS_OK;
}

int oracle_evaluate(const ps_kernel_input* in, uint32_t level, const uint32_t* views, size_t n,
                    const ps_view_state* states, uint32_t geometric, const ps_depth_snapshot* snap, float* const* out,
                    int threads) {
  Scene sc;
  if (!load_scene(in, sc)) return PS_EINVAL;
  set_threads(threads);
  std::vector<std::vector<float>> maps = snapshot_maps(sc, snap);
  for (size_t i = 0; i < n; ++i) {
    State st;
    to_state(states[i], st, true);
    Run r{};
    r.sc = &sc;
    r.view = (int)views[i];
    r.level = (int)level;
    r.geometric = geometric;
    r.topk = sc.cs.topk;
    r.snap = &maps;
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < st.h; ++y)
      for (int x = 0; x < st.w; ++x) eval_pixel(r, st, x, y, 0, 0);
    memcpy(out[i], st.cost.data(), st.cost.size() * sizeof(float));
  }
  return PS_OK;
}

// Rows [y0, y1) only (y1 <= 0: all rows; the other rows of `out` are left as they are): the timing sample of the
// CPU baseline filters the same band of rows it ran.
int oracle_filter_rows(const ps_kernel_input* in, const uint32_t* views, size_t n, const ps_view_state* states,
                       const ps_depth_snapshot* snap, uint8_t* const* out, int threads, int y0, int y1) {
  Scene sc;
  if (!load_scene(in, sc) || !snap) return PS_EINVAL;
  set_threads(threads);
  std::vector<std::vector<float>> maps = snapshot_maps(sc, snap);
  for (size_t i = 0; i < n; ++i) {
    State st;
    to_state(states[i], st, true);
    Run r{};
    r.sc = &sc;
    r.view = (int)views[i];
    r.level = (int)snap->level;
    r.geometric = 1;
    r.topk = sc.cs.topk;
    r.snap = &maps;
    constexpr int CHUNK = 64;
    const int ya = y1 > 0 ? std::max(0, y0) : 0, yb = y1 > 0 ? std::min(st.h, y1) : st.h;
    const int cx = (st.w + CHUNK - 1) / CHUNK;
    const long long items = (long long)std::max(yb - ya, 0) * cx;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long k = 0; k < items; ++k) {
      const int y = ya + (int)(k / cx), xa = (int)(k % cx) * CHUNK, xb = std::min(xa + CHUNK, st.w);
      for (int x = xa; x < xb; ++x) out[i][y * st.w + x] = (uint8_t)filter_pixel(r, st, x, y);
    }
  }
  return PS_OK;
}

int oracle_filter(const ps_kernel_input* in, const uint32_t* views, size_t n, const ps_view_state* states,
                  const ps_depth_snapshot* snap, uint8_t* const* out, int threads) {
  return oracle_filter_rows(in, views, n, states, snap, out, threads, 0, 0);
}

// pm_upsample (patchmatch.cu:741-801), binary32.
int oracle_upsample(const ps_kernel_input* in, uint32_t level, const uint32_t* views, size_t n,
                    const ps_view_state* low, float sigma_s, float sigma_c, ps_view_state* out, int threads) {
  Scene sc;
  if (!load_scene(in, sc) || level < 1) return PS_EINVAL;
  set_threads(threads);
  const float inv2s = 1.0f / (2.0f * sigma_s * sigma_s), inv2c = 1.0f / (2.0f * sigma_c * sigma_c);
  for (size_t i = 0; i < n; ++i) {
    const Img& R = sc.L((int)views[i], (int)level);
    const Img& L = sc.L((int)views[i], (int)level - 1);
    const ps_view_state& lo = low[i];
    ps_view_state& o = out[i];
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < R.h; ++y)
      for (int x = 0; x < R.w; ++x) {
        V3<float> rp = pixel_ray(R, x, y);
        float ip = R.at(x, y);
        float px = ((float)x - 0.5f) * 0.5f, py = ((float)y - 0.5f) * 0.5f;
        int qx0 = (int)roundf(px), qy0 = (int)roundf(py);
        float sw = 0.f, sd = 0.f;
        V3<float> sn = {0.f, 0.f, 0.f};
        float nd = 1e30f, ndep = 0.f;
        V3<float> nn = {0.f, 0.f, 0.f};
        for (int qy = qy0 - 2; qy <= qy0 + 2; ++qy) {
          if (qy < 0 || qy >= L.h) continue;
          for (int qx = qx0 - 2; qx <= qx0 + 2; ++qx) {
            if (qx < 0 || qx >= L.w) continue;
            size_t qi = (size_t)qy * L.w + qx;
            float qw = lo.depth[qi];
            if (!(qw > 0.f)) continue;
            V3<float> nq = {lo.normal[3 * qi], lo.normal[3 * qi + 1], lo.normal[3 * qi + 2]};
            float den = dot3(nq, rp);
            if (!(den < -1e-6f)) continue;
            float d = qw * dot3(nq, pixel_ray(L, qx, qy)) / den;
            if (!(d > 0.f) || !std::isfinite(d)) continue;
            float ds = ((float)qx - px) * ((float)qx - px) + ((float)qy - py) * ((float)qy - py);
            if (ds < nd) {
              nd = ds;
              ndep = d;
              nn = nq;
            }
            float iq = L.at(qx, qy);
            float wgt = ps_expf(-ds * inv2s - (ip - iq) * (ip - iq) * inv2c);
            sw += wgt;
            sd += wgt * d;
            sn.x += wgt * nq.x;
            sn.y += wgt * nq.y;
            sn.z += wgt * nq.z;
          }
        }
        float d = 0.f;
        V3<float> nr = {0.f, 0.f, 0.f};
        bool ok = false;
        if (sw > 1e-12f) {
          d = sd / sw;
          nr = sn;
          ok = true;
        } else if (nd < 1e29f) {
          d = ndep;
          nr = nn;
          ok = true;
        }
        P4 res = {0.f, 0.f, 0.f, 0.f};
        if (ok && dot3(nr, nr) > 1e-24f) {
          nr = nrm3(nr);
          if (dot3(nr, rp) >= 0.f) nr = {-nr.x, -nr.y, -nr.z};
          res = {nr.x, nr.y, nr.z, d};
        }
        size_t p = (size_t)y * R.w + x;
        o.normal[3 * p] = res.x;
        o.normal[3 * p + 1] = res.y;
        o.normal[3 * p + 2] = res.z;
        o.depth[p] = res.w;
        if (o.cost) o.cost[p] = 2.f;
      }
  }
  return PS_OK;
}

// pm_median (patchmatch.cu:805-849), binary32.
int oracle_median(const ps_kernel_input* in, uint32_t level, const uint32_t* views, size_t n,
                  const ps_view_state* inp, ps_view_state* out, int threads) {
  Scene sc;
  if (!load_scene(in, sc)) return PS_EINVAL;
  set_threads(threads);
  for (size_t i = 0; i < n; ++i) {
    const Img& R = sc.L((int)views[i], (int)level);
    const ps_view_state& s = inp[i];
    ps_view_state& o = out[i];
    const int w = R.w, h = R.h;
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < h; ++y)
      for (int x = 0; x < w; ++x) {
        size_t p = (size_t)y * w + x;
        P4 self = {s.normal[3 * p], s.normal[3 * p + 1], s.normal[3 * p + 2], s.depth[p]};
        P4 res = self;
        if (self.w > 0.f) {
          V3<float> rp = pixel_ray(R, x, y);
          float ds[25];
          int qs[25];
          int c = 0;
          for (int qy = std::max(y - 2, 0); qy < std::min(y + 3, h); ++qy)
            for (int qx = std::max(x - 2, 0); qx < std::min(x + 3, w); ++qx) {
              size_t qi = (size_t)qy * w + qx;
              float qw = s.depth[qi];
              if (!(qw > 0.f)) continue;
              V3<float> nq = {s.normal[3 * qi], s.normal[3 * qi + 1], s.normal[3 * qi + 2]};
              float den = dot3(nq, rp);
              if (!(den < -1e-6f)) continue;
              float d = qw * dot3(nq, pixel_ray(R, qx, qy)) / den;
              if (!(d > 0.f) || !std::isfinite(d)) continue;
              int k = c++;
              while (k > 0 && (ds[k - 1] > d || (ds[k - 1] == d && qs[k - 1] > (int)qi))) {
                ds[k] = ds[k - 1];
                qs[k] = qs[k - 1];
                --k;
              }
              ds[k] = d;
              qs[k] = (int)qi;
            }
          if (c > 0) {
            int m = (c - 1) / 2;
            res = {s.normal[3 * qs[m]], s.normal[3 * qs[m] + 1], s.normal[3 * qs[m] + 2], ds[m]};
          }
        }
        o.normal[3 * p] = res.x;
        o.normal[3 * p + 1] = res.y;
        o.normal[3 * p + 2] = res.z;
        o.depth[p] = res.w;
        if (o.cost && s.cost && o.cost != s.cost) o.cost[p] = s.cost[p];
      }
  }
  return PS_OK;
}

// FP64 re-evaluation of given hypotheses: top-K cost of every pixel in binary64 (geometry from FP64 pairs when
// given).  out[i] receives w*h doubles.
int oracle_reeval_f64(const ps_kernel_input* in, uint32_t level, const uint32_t* views, size_t n,
                      const ps_view_state* states, uint32_t geometric, const ps_depth_snapshot* snap,
                      double* const* out, int threads) {
  Scene sc;
  if (!load_scene(in, sc)) return PS_EINVAL;
  set_threads(threads);
  std::vector<std::vector<float>> maps = snapshot_maps(sc, snap);
  for (size_t i = 0; i < n; ++i) {
    State st;
    to_state(states[i], st, true);
    Run r{};
    r.sc = &sc;
    r.view = (int)views[i];
    r.level = (int)level;
    r.geometric = geometric;
    r.topk = sc.cs.topk;
    r.snap = &maps;
    const Img& R = sc.L(r.view, r.level);
#pragma omp parallel for schedule(dynamic, 1)
    for (int y = 0; y < st.h; ++y)
      for (int x = 0; x < st.w; ++x) {
        P4 hh = st.plane[(size_t)y * st.w + x];
        double c = 2.0;
        if (hh.w > 0.f) {
          RS<double> rs = ref_stats<double>(sc, R, x, y);
          c = topk_cost<double>(r, R, rs, x, y, hh);
        }
        out[i][(size_t)y * st.w + x] = c;
      }
  }
  return PS_OK;
}

// ---- known-answer entry points (crates/dense/src/math.rs, kernel.rs, upsample.rs) ----------------------------
uint64_t oracle_mix64(uint64_t z) { return mix64(z); }
uint64_t oracle_rng_state(uint64_t seed, uint64_t key, uint32_t level, uint32_t run, uint32_t t, uint32_t half,
                          uint64_t pixel) {
  return rng_state(seed, key, (int)level, (int)run, (int)t, (int)half, pixel);
}
float oracle_rng_next(uint64_t* state) {
  u64 s = *state;
  float f = rnd(s);
  *state = s;
  return f;
}
uint64_t oracle_hash_bytes(const uint8_t* b, size_t n) {
  uint64_t h = 0xcbf29ce484222325ULL;
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 0x00000100000001b3ULL;
  }
  return h;
}
double oracle_erf(double x) { return ps_erf(x); }
double oracle_emission_norm(double s) { return ps_emission_norm(s); }
double oracle_emission(double c, double s) { return ps_emission(c, s); }
double oracle_visibility_probability(double c, double s) {
  double e = ps_emission(c, s);
  return e / (e + 0.5);
}
// triangulation_prior / incident_prior / resolution_prior (math.rs:84-123)
double oracle_triangulation_prior(double cos_theta, double min_angle_rad) {
  double cmin = cos(min_angle_rad);
  if (cos_theta > cmin) {
    double s = 1.0 - (1.0 - cos_theta) / (1.0 - cmin);
    return std::min(std::max(1.0 - s * s, 0.0), 1.0);
  }
  return 1.0;
}
double oracle_incident_prior(double cos_phi, double sigma) {
  double x = 1.0 - std::max(cos_phi, 0.0);
  return exp(-x * x / (2.0 * sigma * sigma));
}
double oracle_resolution_prior(const double* h, double x, double y, double radius) {
  double c[4][2] = {{x - radius, y - radius}, {x - radius, y + radius}, {x + radius, y + radius}, {x + radius, y - radius}};
  double p[4][2];
  for (int i = 0; i < 4; ++i) {
    double z = h[6] * c[i][0] + h[7] * c[i][1] + h[8];
    p[i][0] = (h[0] * c[i][0] + h[1] * c[i][1] + h[2]) / z;
    p[i][1] = (h[3] * c[i][0] + h[4] * c[i][1] + h[5]) / z;
  }
  double area = 0.0;
  for (int i = 0; i < 4; ++i) area += p[i][0] * p[(i + 1) % 4][1] - p[(i + 1) % 4][0] * p[i][1];
  double a_src = 0.5 * fabs(area), a_ref = (2.0 * radius + 1.0) * (2.0 * radius + 1.0);
  if (a_src <= 0.0 || !std::isfinite(a_src)) return 0.0;
  return std::min(a_src / a_ref, a_ref / a_src);
}
// plane_transfer (math.rs:143-154); returns 1 and writes *out when the transfer exists.
int oracle_plane_transfer(double dq, const double* n, const double* rq, const double* rp, double* out) {
  double num = n[0] * rq[0] + n[1] * rq[1] + n[2] * rq[2];
  double den = n[0] * rp[0] + n[1] * rp[1] + n[2] * rp[2];
  if (den > -1e-6) return 0;
  double d = dq * num / den;
  if (!(d > 0.0 && std::isfinite(d))) return 0;
  *out = d;
  return 1;
}
// num_levels (upsample.rs:35-44)
size_t oracle_num_levels(size_t min_side, size_t max_levels, size_t min_size) {
  size_t l = 1, s = min_side;
  while (l < max_levels && s / 2 >= min_size) {
    s /= 2;
    l += 1;
  }
  return l;
}
// build_pyramid, one step (upsample.rs:46-102): blur3 (σ=0.5, clamped borders), 2×2 average, round to u8.
// out has (w/2)*(h/2) bytes; kout receives the halved intrinsics.
void oracle_pyramid_step(const uint8_t* src, size_t w, size_t h, const double* k, uint8_t* out, double* kout) {
  float g0 = expf(-1.0f / (2.0f * 0.25f));
  float g[3] = {g0, 1.0f, g0};
  float s = g[0] + g[1] + g[2];
  for (float& x : g) x /= s;
  std::vector<float> cur(w * h), tmp(w * h), b(w * h);
  for (size_t i = 0; i < w * h; ++i) cur[i] = (float)src[i];
  for (size_t y = 0; y < h; ++y)
    for (size_t x = 0; x < w; ++x) {
      float a = 0.0f;
      for (int kk = 0; kk < 3; ++kk) {
        long xx = std::min(std::max((long)x + kk - 1, 0L), (long)w - 1);
        a += g[kk] * cur[y * w + xx];
      }
      tmp[y * w + x] = a;
    }
  for (size_t y = 0; y < h; ++y)
    for (size_t x = 0; x < w; ++x) {
      float a = 0.0f;
      for (int kk = 0; kk < 3; ++kk) {
        long yy = std::min(std::max((long)y + kk - 1, 0L), (long)h - 1);
        a += g[kk] * tmp[yy * w + x];
      }
      b[y * w + x] = a;
    }
  size_t nw = w / 2, nh = h / 2;
  for (size_t y = 0; y < nh; ++y)
    for (size_t x = 0; x < nw; ++x) {
      size_t i = 2 * y * w + 2 * x;
      float v = 0.25f * (b[i] + b[i + 1] + b[i + w] + b[i + w + 1]);
      out[y * nw + x] = (uint8_t)std::min(std::max(roundf(v), 0.0f), 255.0f);
    }
  kout[0] = k[0] * 0.5;
  kout[1] = k[1] * 0.5;
  kout[2] = (k[2] + 0.5) * 0.5 - 0.5;
  kout[3] = (k[3] + 0.5) * 0.5 - 0.5;
}
float oracle_expf(float x) { return ps_expf(x); }
double oracle_exp64(double x) { return ps_exp64(x); }
double oracle_acos64(double x) { return ps_acos64(x); }
void oracle_sincosf(float x, float* s, float* c) { ps_sincosf(x, s, c); }

// Footprint bound of the engine's staged source boxes (the half step with PS_TUNE_STAGED; no reference counterpart:
// it decides only where the kernel reads texels from, never a value).  Restates the kernel's per-lane rule: the
// corner taps of the window at (x, y) (radius wr) must be in front of the source (1e-8 < z, zmin < 1e30) and the homography
// terms bounded (Tu, Tv, (|u|+|v|+1)·Tz <= 2^14·zmin, |u|, |v| < 2^14); the lane's texel range is then
// [floor(umin - 1/64), floor(umax + 1/64) + 1] × the same for v.  Returns -1 when the rule rejects the window,
// otherwise the number of taps (window step ws) whose 2×2 texels fall outside that range or whose box address,
// computed as the kernel does (F = u + (1.5·2^23 - lo) rounded toward -inf), differs from floor(u) - lo.  The tap
// positions use the parity build's operation sequence (correctly rounded reciprocal).  range = {lx, hx, ly, hy}.
int oracle_box_footprint_check(const float* H, int x, int y, int wr, int ws, int* range) {
  const float fx = (float)x, fy = (float)y;
  const float sx0 = fx + (float)(-wr), sx1 = fx + (float)wr, sy0 = fy + (float)(-wr), sy1 = fy + (float)wr;
  const float rz0 = std::fma(H[7], sy0, H[8]), rz1 = std::fma(H[7], sy1, H[8]);
  const float z00 = std::fma(H[6], sx0, rz0), z10 = std::fma(H[6], sx1, rz0);
  const float z01 = std::fma(H[6], sx0, rz1), z11 = std::fma(H[6], sx1, rz1);
  if (!(z00 > 1e-8f && z10 > 1e-8f && z01 > 1e-8f && z11 > 1e-8f)) return -1;
  const float rx0 = std::fma(H[1], sy0, H[2]), rx1 = std::fma(H[1], sy1, H[2]);
  const float ry0 = std::fma(H[4], sy0, H[5]), ry1 = std::fma(H[4], sy1, H[5]);
  const float i00 = 1.0f / z00, i10 = 1.0f / z10, i01 = 1.0f / z01, i11 = 1.0f / z11;
  const float u00 = std::fma(H[0], sx0, rx0) * i00, u10 = std::fma(H[0], sx1, rx0) * i10;
  const float u01 = std::fma(H[0], sx0, rx1) * i01, u11 = std::fma(H[0], sx1, rx1) * i11;
  const float v00 = std::fma(H[3], sx0, ry0) * i00, v10 = std::fma(H[3], sx1, ry0) * i10;
  const float v01 = std::fma(H[3], sx0, ry1) * i01, v11 = std::fma(H[3], sx1, ry1) * i11;
  const float umin = std::fmin(std::fmin(u00, u10), std::fmin(u01, u11));
  const float umax = std::fmax(std::fmax(u00, u10), std::fmax(u01, u11));
  const float vmin = std::fmin(std::fmin(v00, v10), std::fmin(v01, v11));
  const float vmax = std::fmax(std::fmax(v00, v10), std::fmax(v01, v11));
  const float zmin = std::fmin(std::fmin(z00, z10), std::fmin(z01, z11));
  const float mx = std::fmax(std::fabs(sx0), std::fabs(sx1)), my = std::fmax(std::fabs(sy0), std::fabs(sy1));
  const float tu = std::fabs(H[0]) * mx + std::fabs(H[1]) * my + std::fabs(H[2]);
  const float tv = std::fabs(H[3]) * mx + std::fabs(H[4]) * my + std::fabs(H[5]);
  const float tz = std::fabs(H[6]) * mx + std::fabs(H[7]) * my + std::fabs(H[8]);
  const float ua = std::fmax(std::fabs(umin), std::fabs(umax)), va = std::fmax(std::fabs(vmin), std::fabs(vmax));
  const float lim = 16384.0f * zmin;
  if (!(zmin < 1e30f && tu <= lim && tv <= lim && (ua + va + 1.0f) * tz <= lim && ua < 16384.0f && va < 16384.0f))
    return -1;
  const int lx = (int)std::floor(umin - 0.015625f), hx = (int)std::floor(umax + 0.015625f) + 1;
  const int ly = (int)std::floor(vmin - 0.015625f), hy = (int)std::floor(vmax + 0.015625f) + 1;
  range[0] = lx;
  range[1] = hx;
  range[2] = ly;
  range[3] = hy;
  const float mxb = 12582912.0f - (float)lx, myb = 12582912.0f - (float)ly;
  uint32_t mbits;
  const float mag = 12582912.0f;
  std::memcpy(&mbits, &mag, 4);
  const int wn = (2 * wr) / ws + 1;
  int bad = 0;
  for (int a = 0; a < wn; ++a) {
    const int dy = -wr + a * ws;
    const float sy = fy + (float)dy;
    const float rx = std::fma(H[1], sy, H[2]), ry = std::fma(H[4], sy, H[5]), rz = std::fma(H[7], sy, H[8]);
    for (int b = 0; b < wn; ++b) {
      const int dx = -wr + b * ws;
      const float sx = fx + (float)dx;
      const float izz = 1.0f / std::fma(H[6], sx, rz);
      const float u = std::fma(H[0], sx, rx) * izz, v = std::fma(H[3], sx, ry) * izz;
      const float xf = std::floor(u), yf = std::floor(v);
      if (!(xf >= (float)lx && xf + 1.0f <= (float)hx && yf >= (float)ly && yf + 1.0f <= (float)hy)) {
        bad++;
        continue;
      }
      // u + mxb and v + myb are exact in binary64; rounding toward -inf onto the integer grid of [2^23, 2^24)
      const float Fu = (float)std::floor((double)u + (double)mxb), Fv = (float)std::floor((double)v + (double)myb);
      uint32_t bu, bv;
      std::memcpy(&bu, &Fu, 4);
      std::memcpy(&bv, &Fv, 4);
      if ((int)(bu - mbits) != (int)xf - lx || (int)(bv - mbits) != (int)yf - ly || Fu - mxb != xf || Fv - myb != yf)
        bad++;
    }
  }
  return bad;
}


// ================================================================================================ post-processing
// remove_speckles (crates/dense/src/postproc.rs:77-129): depth-first growth from every unlabelled valid pixel in
// row-major order over 4-neighbours with |d_j - d_i| <= rel·min(d_i, d_j); a component smaller than
// ceil(w·h·frac) whose lower median cost (costs sorted by total order, element len/2) exceeds keep is erased
// (depth 0, normal 0).  normal: 3 floats per pixel.
// fill_holes (crates/dense/src/postproc.rs:139-201): every invalid pixel whose own (raw) cost is at most max_cost
// walks the 8 directions up to maxd = max(round(diag · max_frac), 1) steps over the 8-bit gray image, stopping at the
// border or where the gray value jumps by more than step = (int)(edge_step · 255) from the previous pixel, and takes
// the valid pixel it meets with the smallest (|gray difference|, distance) (the first direction on ties); its plane
// is transferred to the pixel (plane_transfer).  Fills read the unfilled state only and are applied at the end.
int oracle_fill_holes(float* depth, float* normal, float* cost, const float* raw_cost, const uint8_t* gray,
                      const double* k, uint32_t w, uint32_t h, double max_frac, float edge_step, float max_cost,
                      uint64_t* filled) {
  if (!depth || !normal || !cost || !raw_cost || !gray || !k) return PS_EINVAL;
  const long long W = w, H = h;
  const long long maxd = std::max<long long>((long long)std::round(std::sqrt((double)(W * W + H * H)) * max_frac), 1);
  const int step = (int)(edge_step * 255.0f);
  const size_t n = (size_t)w * h;
  std::vector<char> valid(n);
  for (size_t i = 0; i < n; ++i) valid[i] = depth[i] > 0.0f;
  struct Fill {
    size_t i;
    float d, nx, ny, nz, c;
  };
  std::vector<Fill> fills;
  static const int dirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {1, -1}, {-1, 1}};
  for (long long y = 0; y < H; ++y)
    for (long long x = 0; x < W; ++x) {
      const size_t i = (size_t)(y * W + x);
      if (valid[i] || raw_cost[i] > max_cost) continue;
      const int ip = gray[i];
      bool found = false;
      int bdiff = 0;
      long long bs = 0;
      size_t bq = 0;
      for (int d = 0; d < 8; ++d) {
        int prev = ip;
        for (long long st = 1; st <= maxd; ++st) {
          const long long qx = x + dirs[d][0] * st, qy = y + dirs[d][1] * st;
          if (qx < 0 || qy < 0 || qx >= W || qy >= H) break;
          const size_t q = (size_t)(qy * W + qx);
          const int iq = gray[q];
          if (std::abs(iq - prev) > step) break;
          prev = iq;
          if (valid[q]) {
            const int diff = std::abs(iq - ip);
            if (!found || diff < bdiff || (diff == bdiff && st < bs)) {
              found = true;
              bdiff = diff;
              bs = st;
              bq = q;
            }
            break;
          }
        }
      }
      if (!found) continue;
      const double nq[3] = {(double)normal[3 * bq], (double)normal[3 * bq + 1], (double)normal[3 * bq + 2]};
      const double qx = (double)(bq % w), qy = (double)(bq / w);
      const double rq[3] = {(qx - k[2]) / k[0], (qy - k[3]) / k[1], 1.0};
      const double rp[3] = {((double)x - k[2]) / k[0], ((double)y - k[3]) / k[1], 1.0};
      double dd;
      if (oracle_plane_transfer((double)depth[bq], nq, rq, rp, &dd))
        fills.push_back({i, (float)dd, normal[3 * bq], normal[3 * bq + 1], normal[3 * bq + 2], cost[bq]});
    }
  for (const Fill& f : fills) {
    depth[f.i] = f.d;
    normal[3 * f.i] = f.nx;
    normal[3 * f.i + 1] = f.ny;
    normal[3 * f.i + 2] = f.nz;
    cost[f.i] = f.c;
  }
  if (filled) *filled = fills.size();
  return PS_OK;
}

int oracle_remove_speckles(float* depth, float* normal, const float* cost, uint32_t w, uint32_t h, float rel,
                           double frac, float keep, uint64_t* removed) {
  if (!depth || !normal || !cost) return PS_EINVAL;
  const size_t n = (size_t)w * h;
  const size_t min_area = (size_t)std::ceil((double)n * frac);
  if (removed) *removed = 0;
  if (min_area <= 1) return PS_OK;
  std::vector<uint32_t> label(n, UINT32_MAX);
  std::vector<size_t> stack, comp;
  std::vector<float> costs;
  uint64_t erased = 0;
  auto total_less = [](float a, float b) {  // f32::total_cmp
    int32_t ia, ib;
    memcpy(&ia, &a, 4);
    memcpy(&ib, &b, 4);
    ia ^= (int32_t)((uint32_t)(ia >> 31) >> 1);
    ib ^= (int32_t)((uint32_t)(ib >> 31) >> 1);
    return ia < ib;
  };
  for (size_t start = 0; start < n; ++start) {
    if (depth[start] <= 0.0f || label[start] != UINT32_MAX) continue;
    comp.clear();
    stack.push_back(start);
    label[start] = (uint32_t)start;
    while (!stack.empty()) {
      const size_t i = stack.back();
      stack.pop_back();
      comp.push_back(i);
      const size_t x = i % w, y = i / w;
      const float di = depth[i];
      size_t nb[4] = {SIZE_MAX, SIZE_MAX, SIZE_MAX, SIZE_MAX};
      if (x > 0) nb[0] = i - 1;
      if (x + 1 < w) nb[1] = i + 1;
      if (y > 0) nb[2] = i - w;
      if (y + 1 < h) nb[3] = i + w;
      for (size_t j : nb) {
        if (j == SIZE_MAX || label[j] != UINT32_MAX || depth[j] <= 0.0f) continue;
        if (std::fabs(depth[j] - di) <= rel * std::min(di, depth[j])) {
          label[j] = (uint32_t)start;
          stack.push_back(j);
        }
      }
    }
    if (comp.size() < min_area) {
      costs.clear();
      for (size_t i : comp) costs.push_back(cost[i]);
      std::sort(costs.begin(), costs.end(), total_less);
      if (costs[costs.size() / 2] > keep) {
        for (size_t i : comp) {
          depth[i] = 0.0f;
          normal[3 * i] = normal[3 * i + 1] = normal[3 * i + 2] = 0.0f;
        }
        erased += comp.size();
      }
    }
  }
  if (removed) *removed = erased;
  return PS_OK;
}

// Consistency fusion (crates/dense/src/fusion.rs:219-459, residual handling "none", colour = gray u8 of `img`).
// Views in index order (used[v] != 0); within a view every pixel is evaluated independently (rows in parallel, the
// result does not depend on it).  Points are written in the reference's order into caller buffers of `capacity`
// points; vis holds vis_stride entries per point.  Returns the point count in *count.
namespace {
struct FCam {
  double k[4], r[9], t[3], baseline;
  int w, h;
};
void f_backproject(const FCam& c, double col, double row, double d, double* X) {
  const double cc[3] = {(col - c.k[2]) / c.k[0] * d, (row - c.k[3]) / c.k[1] * d, d};
  const double p[3] = {cc[0] - c.t[0], cc[1] - c.t[1], cc[2] - c.t[2]};
  X[0] = c.r[0] * p[0] + c.r[3] * p[1] + c.r[6] * p[2];
  X[1] = c.r[1] * p[0] + c.r[4] * p[1] + c.r[7] * p[2];
  X[2] = c.r[2] * p[0] + c.r[5] * p[1] + c.r[8] * p[2];
}
bool f_project(const FCam& c, const double* x, double* u, double* v, double* z) {
  const double cz = c.r[6] * x[0] + c.r[7] * x[1] + c.r[8] * x[2] + c.t[2];
  if (cz <= 0.0) return false;
  const double cx = c.r[0] * x[0] + c.r[1] * x[1] + c.r[2] * x[2] + c.t[0];
  const double cy = c.r[3] * x[0] + c.r[4] * x[1] + c.r[5] * x[2] + c.t[1];
  *u = c.k[0] * cx / cz + c.k[2];
  *v = c.k[1] * cy / cz + c.k[3];
  *z = cz;
  return true;
}
void f_normal(const FCam& c, const float* n3, double* n) {
  const double m[3] = {(double)n3[0], (double)n3[1], (double)n3[2]};
  n[0] = c.r[0] * m[0] + c.r[3] * m[1] + c.r[6] * m[2];
  n[1] = c.r[1] * m[0] + c.r[4] * m[1] + c.r[7] * m[2];
  n[2] = c.r[2] * m[0] + c.r[5] * m[1] + c.r[8] * m[2];
}
double f_inv_var(const ps_fusion_params& p, const FCam& c, double d, float cost) {
  if (!p.inverse_variance || !(c.baseline > 0.0)) return 1.0;
  const double spx = p.sigma_px0 + p.sigma_px_slope * (double)std::min(std::max(cost, 0.0f), 2.0f);
  const double sd = d * d * spx / (c.k[0] * c.baseline);
  return 1.0 / std::max(sd * sd, 1e-300);
}
double f_gray(const float* img, const FCam& c, int col, int row) {
  const int x = std::min(col, c.w - 1), y = std::min(row, c.h - 1);
  const float v = img[(size_t)y * c.w + x] * 255.0f;
  return (double)(uint8_t)std::min(std::max(std::nearbyint(v), 0.0f), 255.0f);
}
struct FPoint {
  float pos[3], nrm[3];
  uint8_t col[3];
  uint64_t key;
  std::vector<uint16_t> vis;
};
// filter_visibility's test of one point (crates/dense/src/visibility.rs:117-138): candidate views are the overlap
// lists of its views in order, de-duplicated, cut at check_views; a view whose depth lies behind the point by more
// than tau is a violation, one within tau a support.
bool visibility_violated(const float* pos, const uint16_t* vis, size_t nvis, uint32_t nviews,
                         const ps_fusion_view* cams, const std::vector<FCam>& fc, const float* const* depth,
                         const uint8_t* used, uint32_t check_views, uint32_t min_violations, double tau) {
  const double x[3] = {(double)pos[0], (double)pos[1], (double)pos[2]};
  std::vector<int> cand;
  bool full = false;
  for (size_t t = 0; t < nvis; ++t) {
    const uint16_t v = vis[t];
    if (full) break;
    if (v >= nviews) continue;
    for (uint32_t j = 0; j < cams[v].num_overlap; ++j) {
      if (cand.size() >= check_views) {
        full = true;
        break;
      }
      const int o = (int)cams[v].overlap[j];
      if (std::find(cand.begin(), cand.end(), o) == cand.end()) cand.push_back(o);
    }
  }
  int viol = 0, sup = 0;
  for (int v : cand) {
    if (v < 0 || v >= (int)nviews || !used[v]) continue;
    const FCam& c = fc[v];
    const double cx = c.r[0] * x[0] + c.r[1] * x[1] + c.r[2] * x[2] + c.t[0];
    const double cy = c.r[3] * x[0] + c.r[4] * x[1] + c.r[5] * x[2] + c.t[1];
    const double cz = c.r[6] * x[0] + c.r[7] * x[1] + c.r[8] * x[2] + c.t[2];
    if (cz <= 0.0) continue;
    const double col = std::round(c.k[0] * cx / cz + c.k[2]), row = std::round(c.k[1] * cy / cz + c.k[3]);
    if (col < 0.0 || row < 0.0 || col >= (double)c.w || row >= (double)c.h) continue;
    const double dv = (double)depth[v][(size_t)row * c.w + (size_t)col];
    if (dv <= 0.0) continue;
    if (cz < dv * (1.0 - tau))
      viol++;
    else if (std::fabs(cz - dv) <= tau * dv)
      sup++;
  }
  return viol >= (int)min_violations && viol > sup;
}

// scene_gsd (crates/dense/src/fusion.rs:463-487): per used view the median of every 97th valid depth over fx, then
// the median over views (medians interpolated at 0.5·(n-1)); 0 without valid depths.
double scene_gsd(uint32_t nviews, const std::vector<FCam>& fc, const float* const* depth, const uint8_t* used) {
  auto median = [](std::vector<double>& a) {
    std::sort(a.begin(), a.end());
    const double pos = 0.5 * (double)(a.size() - 1);
    const size_t lo = (size_t)std::floor(pos), hi = std::min(lo + 1, a.size() - 1);
    return a[lo] + (a[hi] - a[lo]) * (pos - (double)lo);
  };
  std::vector<double> gs;
  for (uint32_t v = 0; v < nviews; ++v) {
    if (!used[v]) continue;
    std::vector<double> dd;
    size_t k = 0;
    for (size_t i = 0; i < (size_t)fc[v].w * fc[v].h; ++i)
      if (depth[v][i] > 0.0f) {
        if (k % 97 == 0) dd.push_back((double)depth[v][i]);
        ++k;
      }
    if (!dd.empty()) gs.push_back(median(dd) / fc[v].k[0]);
  }
  return gs.empty() ? 0.0 : median(gs);
}

// smooth_along_normals (crates/dense/src/smooth.rs:143-220) over points in cloud order: Jacobi passes; each point
// sums its neighbours within the radius in the order of the 27 cells around it ((z, y, x) offsets), each cell's points
// in cloud order.  Returns the median absolute displacement of the last pass (0 when nothing ran).
double smooth_points(std::vector<float*>& pos, const std::vector<const float*>& nrm3, double gsd, uint32_t iterations,
                     double radius_gsd, double sigma_range_gsd, double normal_deg) {
  const size_t n = pos.size();
  if (!(iterations > 0 && radius_gsd > 0.0 && sigma_range_gsd > 0.0) || gsd <= 0.0 || n == 0) return 0.0;
  const double r = radius_gsd * gsd;
  const double r2 = r * r;
  const double inv_2ss = 1.0 / (2.0 * ((0.5 * r) * (0.5 * r)));
  const double sr = sigma_range_gsd * gsd;
  const double inv_2sr = 1.0 / (2.0 * (sr * sr));
  const double cos_n = std::cos(ps_to_radians_f64(normal_deg));
  std::vector<std::array<double, 3>> nrm(n);
  for (size_t i = 0; i < n; ++i) {
    const double m[3] = {(double)nrm3[i][0], (double)nrm3[i][1], (double)nrm3[i][2]};
    const double l = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    nrm[i] = l > 1e-12 ? std::array<double, 3>{m[0] / l, m[1] / l, m[2] / l} : std::array<double, 3>{0.0, 0.0, 0.0};
  }
  double last = 0.0;
  for (uint32_t it = 0; it < iterations; ++it) {
    // cell -> points in cloud order (cells packed 21 bits per axis around 2^20; the device requires that range)
    auto pack = [](long long x, long long y, long long z) {
      return ((uint64_t)(x + (1ll << 20)) << 42) | ((uint64_t)(y + (1ll << 20)) << 21) | (uint64_t)(z + (1ll << 20));
    };
    std::unordered_map<uint64_t, std::vector<uint32_t>> grid;
    grid.reserve(n);
    std::vector<std::array<long long, 3>> cell(n);
    for (size_t i = 0; i < n; ++i) {
      for (int a = 0; a < 3; ++a) cell[i][a] = (long long)std::floor((double)pos[i][a] / r);
      grid[pack(cell[i][0], cell[i][1], cell[i][2])].push_back((uint32_t)i);
    }
    std::vector<std::array<float, 3>> next(n);
    std::vector<double> disp(n);
#pragma omp parallel for schedule(dynamic, 256)
    for (long long ii = 0; ii < (long long)n; ++ii) {
      const size_t i = (size_t)ii;
      const double pi[3] = {(double)pos[i][0], (double)pos[i][1], (double)pos[i][2]};
      const auto& ni = nrm[i];
      double t = 0.0;
      if (!(ni[0] == 0.0 && ni[1] == 0.0 && ni[2] == 0.0)) {
        double sw = 1.0, swd = 0.0;
        for (long long dz = -1; dz <= 1; ++dz)
          for (long long dy = -1; dy <= 1; ++dy)
            for (long long dx = -1; dx <= 1; ++dx) {
              auto g = grid.find(pack(cell[i][0] + dx, cell[i][1] + dy, cell[i][2] + dz));
              if (g == grid.end()) continue;
              for (uint32_t j : g->second) {
                const double dv[3] = {(double)pos[j][0] - pi[0], (double)pos[j][1] - pi[1], (double)pos[j][2] - pi[2]};
                const double d2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
                if (d2 > r2 || j == i) continue;
                const auto& nj = nrm[j];
                if (ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2] < cos_n) continue;
                const double dn = ni[0] * dv[0] + ni[1] * dv[1] + ni[2] * dv[2];
                const double w = ps_exp64(-d2 * inv_2ss - dn * dn * inv_2sr);
                sw += w;
                swd += w * dn;
              }
            }
        t = swd / sw;
      }
      for (int a = 0; a < 3; ++a) next[i][a] = (float)(pi[a] + t * ni[a]);
      disp[i] = std::fabs(t);
    }
    for (size_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) pos[i][a] = next[i][a];
    std::sort(disp.begin(), disp.end());  // median_in_place (crates/dense/src/math.rs:126-141)
    const double q = 0.5 * (double)(n - 1);
    const size_t lo = (size_t)std::floor(q), hi = std::min(lo + 1, n - 1);
    last = disp[lo] + (disp[hi] - disp[lo]) * (q - (double)lo);
  }
  return last;
}
}  // namespace

int oracle_fuse(uint32_t nviews, const ps_fusion_view* cams, const uint32_t* widths, const uint32_t* heights,
                const float* const* depth, const float* const* normal, const float* const* cost,
                const float* const* img, const uint8_t* used, const ps_fusion_params* p, int threads,
                uint64_t capacity, float* positions, float* normals, uint8_t* colors, uint64_t* keys,
                uint8_t* vis_counts, uint16_t* vis, uint32_t vis_stride, uint64_t* count, uint64_t* residual_count,
                uint64_t* visibility_removed) {
  if (!cams || !widths || !heights || !depth || !normal || !cost || !img || !used || !p || !count) return PS_EINVAL;
  if (p->residual > PS_FUSION_RESIDUAL_SECOND_PASS) return PS_EINVAL;
  set_threads(threads);
  std::vector<FCam> fc(nviews);
  for (uint32_t v = 0; v < nviews; ++v) {
    memcpy(fc[v].k, cams[v].k, sizeof fc[v].k);
    memcpy(fc[v].r, cams[v].r, sizeof fc[v].r);
    memcpy(fc[v].t, cams[v].t, sizeof fc[v].t);
    fc[v].baseline = cams[v].baseline;
    fc[v].w = (int)widths[v];
    fc[v].h = (int)heights[v];
  }
  const bool second = p->residual == PS_FUSION_RESIDUAL_SECOND_PASS;
  std::vector<std::vector<uint8_t>> marks(nviews), consumed(nviews);
  for (uint32_t v = 0; v < nviews; ++v)
    if (used[v]) {
      marks[v].assign((size_t)fc[v].w * fc[v].h, 0);
      if (second) consumed[v].assign((size_t)fc[v].w * fc[v].h, 0);
    }
  std::vector<std::vector<int>> ovs(nviews);
  for (uint32_t v = 0; v < nviews; ++v) {
    if (!used[v]) continue;
    for (uint32_t j = 0; j < cams[v].num_overlap && ovs[v].size() < p->consistency_num_images; ++j) {
      const uint32_t o = cams[v].overlap[j];
      if (o < nviews && used[o] && o != v) ovs[v].push_back((int)o);
    }
  }
  const double r2 = p->max_reproj_error * p->max_reproj_error;
  // ConsCtx::evaluate (fusion.rs:390-460): the weighted mean point of the reference pixel and the agreeing pixels of
  // its overlap views under the tolerances (depth_tol, cos_n); false when the normal sum vanishes.
  auto evaluate = [&](uint32_t v, int row, int col, double depth_tol, double cos_n,
                      std::vector<std::pair<int, int>>& hits, FPoint& pt) -> bool {
    const FCam& cv = fc[v];
    const size_t pix = (size_t)row * cv.w + col;
    const double d = (double)depth[v][pix];
    double x[3], nw[3];
    f_backproject(cv, (double)col, (double)row, d, x);
    f_normal(cv, normal[v] + 3 * pix, nw);
    const double w0 = f_inv_var(*p, cv, d, cost[v][pix]);
    double sw = w0;
    double sx[3] = {x[0] * w0, x[1] * w0, x[2] * w0};
    double sn[3] = {nw[0] * w0, nw[1] * w0, nw[2] * w0};
    const double c0 = f_gray(img[v], cv, col, row);
    double sc[3] = {c0 * w0, c0 * w0, c0 * w0};
    hits.clear();
    for (int o : ovs[v]) {
      const FCam& oc = fc[o];
      double u, vv, z;
      if (!f_project(oc, x, &u, &vv, &z)) continue;
      const double cu = std::floor(u + 0.5), rv = std::floor(vv + 0.5);
      if (cu < 0.0 || rv < 0.0 || cu >= (double)oc.w || rv >= (double)oc.h) continue;
      const size_t opix = (size_t)rv * oc.w + (size_t)cu;
      const double od = (double)depth[o][opix];
      if (od <= 0.0 || std::fabs(z - od) / od > depth_tol) continue;
      double xo[3];
      f_backproject(oc, cu, rv, od, xo);
      double bu, bv, bz;
      if (!f_project(cv, xo, &bu, &bv, &bz)) continue;
      const double eu = bu - (double)col, ev = bv - (double)row;
      if (eu * eu + ev * ev > r2) continue;
      double no[3];
      f_normal(oc, normal[o] + 3 * opix, no);
      if (no[0] * nw[0] + no[1] * nw[1] + no[2] * nw[2] < cos_n) continue;
      const double co = f_gray(img[o], oc, (int)cu, (int)rv);
      const double wo = f_inv_var(*p, oc, od, cost[o][opix]);
      sw += wo;
      for (int k = 0; k < 3; ++k) {
        sx[k] += wo * xo[k];
        sn[k] += wo * no[k];
        sc[k] += wo * co;
      }
      hits.push_back({o, (int)opix});
    }
    const double m = sw;
    const double l = std::sqrt(sn[0] * sn[0] + sn[1] * sn[1] + sn[2] * sn[2]);
    if (l < 1.1920928955078125e-07) return false;
    for (int k = 0; k < 3; ++k) {
      pt.pos[k] = (float)(sx[k] / m);
      pt.nrm[k] = (float)(sn[k] / l);
      pt.col[k] = (uint8_t)std::round(sc[k] / m);
    }
    pt.key = ((uint64_t)cams[v].image_id << 32) | ((uint64_t)(row & 0xffff) << 16) | (uint64_t)(col & 0xffff);
    pt.vis.assign(1, (uint16_t)v);
    for (auto& hq : hits) pt.vis.push_back((uint16_t)hq.first);
    std::sort(pt.vis.begin(), pt.vis.end());
    pt.vis.erase(std::unique(pt.vis.begin(), pt.vis.end()), pt.vis.end());
    return true;
  };
  // first pass (fusion.rs:243-333): views in index order, pixels independent within a view
  const double cos_n = std::cos(ps_to_radians_f64(p->max_normal_error_deg));
  std::vector<FPoint> out1, out2;
  for (uint32_t v = 0; v < nviews; ++v) {
    if (!used[v]) continue;
    const FCam& cv = fc[v];
    std::vector<std::vector<FPoint>> rows(cv.h);
#pragma omp parallel for schedule(dynamic, 4)
    for (int row = 0; row < cv.h; ++row) {
      std::vector<std::pair<int, int>> hits;
      for (int col = 0; col < cv.w; ++col) {
        const size_t pix = (size_t)row * cv.w + col;
        if (depth[v][pix] <= 0.0f) continue;
        if (p->mark_used && __atomic_load_n(&marks[v][pix], __ATOMIC_RELAXED) != 0) continue;
        FPoint pt;
        const bool okp = evaluate(v, row, col, p->max_depth_error, cos_n, hits, pt);
        if (hits.size() < p->min_consistent_views || !okp) continue;
        if (p->mark_used) {
          for (auto& hq : hits) {
            const FCam& oc = fc[hq.first];
            if (p->mark_radius == 0) {
              __atomic_store_n(&marks[hq.first][hq.second], (uint8_t)1, __ATOMIC_RELAXED);
              continue;
            }
            const int cx0 = hq.second % oc.w, cy0 = hq.second / oc.w, r = (int)p->mark_radius;
            const double d0 = (double)depth[hq.first][hq.second];
            for (int yy = std::max(cy0 - r, 0); yy <= std::min(cy0 + r, oc.h - 1); ++yy)
              for (int xx = std::max(cx0 - r, 0); xx <= std::min(cx0 + r, oc.w - 1); ++xx) {
                const size_t qq = (size_t)yy * oc.w + xx;
                const double dq = (double)depth[hq.first][qq];
                if (dq > 0.0 && std::fabs(dq - d0) <= p->max_depth_error * d0)
                  __atomic_store_n(&marks[hq.first][qq], (uint8_t)1, __ATOMIC_RELAXED);
              }
          }
        }
        if (second) {
          __atomic_store_n(&consumed[v][pix], (uint8_t)1, __ATOMIC_RELAXED);
          for (auto& hq : hits) __atomic_store_n(&consumed[hq.first][hq.second], (uint8_t)1, __ATOMIC_RELAXED);
        }
        rows[row].push_back(std::move(pt));
      }
    }
    for (auto& r : rows)
      for (auto& pt : r) out1.push_back(std::move(pt));
  }
  if (second) {
    // second_pass (fusion.rs:540-627)
    const double dtol2 = std::isnan(p->residual_depth_error) ? 0.5 * p->max_depth_error : p->residual_depth_error;
    const double ndeg2 =
        std::isnan(p->residual_normal_error_deg) ? 0.67 * p->max_normal_error_deg : p->residual_normal_error_deg;
    const double cos2 = std::cos(ps_to_radians_f64(ndeg2));
    // depth_gsd (fusion.rs:469-487): per used view the median of every 97th valid depth (row-major) over fx, then
    // the median of those; median = quantile_sorted(·, 0.5)
    auto median = [](std::vector<double>& a) {
      std::sort(a.begin(), a.end());
      const double pos = 0.5 * (double)(a.size() - 1);
      const size_t lo = (size_t)std::floor(pos), hi = std::min(lo + 1, a.size() - 1);
      return a[lo] + (a[hi] - a[lo]) * (pos - (double)lo);
    };
    std::vector<double> gs;
    for (uint32_t v = 0; v < nviews; ++v) {
      if (!used[v]) continue;
      std::vector<double> dd;
      size_t k = 0;
      for (size_t i = 0; i < (size_t)fc[v].w * fc[v].h; ++i)
        if (depth[v][i] > 0.0f) {
          if (k % 97 == 0) dd.push_back((double)depth[v][i]);
          ++k;
        }
      if (dd.empty()) continue;
      gs.push_back(median(dd) / fc[v].k[0]);
    }
    const double gsd = gs.empty() ? 0.0 : median(gs);
    const double min_dist = p->residual_min_dist_gsd * gsd;
    // exact neighbourhood test of first-pass points: cells of size min_dist, the 27 cells around
    std::map<std::array<long long, 3>, std::vector<uint32_t>> grid;
    auto cell_of = [&](const float* x) {
      return std::array<long long, 3>{(long long)std::floor((double)x[0] / min_dist),
                                      (long long)std::floor((double)x[1] / min_dist),
                                      (long long)std::floor((double)x[2] / min_dist)};
    };
    if (min_dist > 0.0)
      for (uint32_t i = 0; i < out1.size(); ++i) grid[cell_of(out1[i].pos)].push_back(i);
    auto any_within = [&](const float* x) {
      const auto c = cell_of(x);
      const double rr = min_dist * min_dist;
      for (long long dz = -1; dz <= 1; ++dz)
        for (long long dy = -1; dy <= 1; ++dy)
          for (long long dx = -1; dx <= 1; ++dx) {
            auto it = grid.find({c[0] + dx, c[1] + dy, c[2] + dz});
            if (it == grid.end()) continue;
            for (uint32_t i : it->second) {
              const float* q = out1[i].pos;
              double d2 = 0.0;
              for (int a2 = 0; a2 < 3; ++a2) {
                const double t = (double)q[a2] - (double)x[a2];
                d2 = d2 + t * t;
              }
              if (d2 <= rr) return true;
            }
          }
      return false;
    };
    std::vector<uint64_t> offset(nviews + 1, 0);
    for (uint32_t v = 0; v < nviews; ++v)
      offset[v + 1] = offset[v] + (used[v] ? (uint64_t)fc[v].w * fc[v].h : 0);
    if (offset[nviews] >= 0xffffffffull) return PS_EINVAL;
    std::vector<std::vector<uint32_t>> owner(nviews);
    for (uint32_t v = 0; v < nviews; ++v)
      if (used[v]) owner[v].assign((size_t)fc[v].w * fc[v].h, 0xffffffffu);
    struct Cand {
      uint32_t v;
      size_t pix;
      FPoint pt;
    };
    // stage 1 in parallel over rows (the ownership is an atomic minimum, so the order does not matter); candidates
    // are collected per row and visited in (view, row, column) order afterwards
    auto fetch_min = [](uint32_t* a, uint32_t v) {
      uint32_t cur = __atomic_load_n(a, __ATOMIC_RELAXED);
      while (v < cur && !__atomic_compare_exchange_n(a, &cur, v, true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
      }
    };
    std::vector<std::vector<std::vector<Cand>>> cands(nviews);
    for (uint32_t v = 0; v < nviews; ++v) {
      if (!used[v]) continue;
      const FCam& cv = fc[v];
      cands[v].resize(cv.h);
#pragma omp parallel for schedule(dynamic, 4)
      for (int row = 0; row < cv.h; ++row) {
        std::vector<std::pair<int, int>> hits;
        for (int col = 0; col < cv.w; ++col) {
          const size_t pix = (size_t)row * cv.w + col;
          if (depth[v][pix] <= 0.0f || consumed[v][pix] != 0) continue;
          FPoint pt;
          if (!evaluate(v, row, col, dtol2, cos2, hits, pt)) continue;
          if (hits.size() < p->residual_min_views) continue;
          if (min_dist > 0.0 && any_within(pt.pos)) continue;
          const uint32_t id = (uint32_t)(offset[v] + pix);
          fetch_min(&owner[v][pix], id);
          for (auto& hq : hits) fetch_min(&owner[hq.first][hq.second], id);
          cands[v][row].push_back({v, pix, std::move(pt)});
        }
      }
    }
    for (auto& cv : cands)
      for (auto& cr : cv)
        for (auto& c : cr)
          if (owner[c.v][c.pix] == (uint32_t)(offset[c.v] + c.pix)) out2.push_back(std::move(c.pt));
  }
  // filter_visibility (crates/dense/src/visibility.rs:106-151) over both passes' points, order kept
  uint64_t vis_removed = 0;
  if (p->visibility_check_views > 0 && p->visibility_tau > 0.0 && p->visibility_min_violations > 0) {
    for (std::vector<FPoint>* part : {&out1, &out2}) {
      std::vector<FPoint> kept;
      for (auto& pt : *part) {
        if (visibility_violated(pt.pos, pt.vis.data(), pt.vis.size(), nviews, cams, fc, depth, used,
                                p->visibility_check_views, p->visibility_min_violations, p->visibility_tau)) {
          vis_removed++;
          continue;
        }
        kept.push_back(std::move(pt));
      }
      *part = std::move(kept);
    }
  }
  if (visibility_removed) *visibility_removed = vis_removed;
  // smooth_along_normals (crates/dense/src/smooth.rs:143-220) over the cloud in its order (first pass, then second)
  if (p->smooth_iterations > 0 && p->smooth_radius_gsd > 0.0 && p->smooth_sigma_range_gsd > 0.0) {
    std::vector<FPoint*> cl;
    for (auto& pt : out1) cl.push_back(&pt);
    for (auto& pt : out2) cl.push_back(&pt);
    auto median = [](std::vector<double>& a) {
      std::sort(a.begin(), a.end());
      const double pos = 0.5 * (double)(a.size() - 1);
      const size_t lo = (size_t)std::floor(pos), hi = std::min(lo + 1, a.size() - 1);
      return a[lo] + (a[hi] - a[lo]) * (pos - (double)lo);
    };
    std::vector<double> gs;  // scene_gsd (fusion.rs:463-487)
    for (uint32_t v = 0; v < nviews; ++v) {
      if (!used[v]) continue;
      std::vector<double> dd;
      size_t k = 0;
      for (size_t i = 0; i < (size_t)fc[v].w * fc[v].h; ++i)
        if (depth[v][i] > 0.0f) {
          if (k % 97 == 0) dd.push_back((double)depth[v][i]);
          ++k;
        }
      if (!dd.empty()) gs.push_back(median(dd) / fc[v].k[0]);
    }
    const double gsd = gs.empty() ? 0.0 : median(gs);
    std::vector<float*> ppos;
    std::vector<const float*> pnrm;
    for (FPoint* q : cl) {
      ppos.push_back(q->pos);
      pnrm.push_back(q->nrm);
    }
    smooth_points(ppos, pnrm, gsd, p->smooth_iterations, p->smooth_radius_gsd, p->smooth_sigma_range_gsd,
                  p->smooth_normal_deg);
  }
  uint64_t n_out = 0;
  for (std::vector<FPoint>* part : {&out1, &out2})
    for (auto& pt : *part) {
      if (n_out < capacity) {
        if (positions) memcpy(positions + 3 * n_out, pt.pos, 12);
        if (normals) memcpy(normals + 3 * n_out, pt.nrm, 12);
        if (colors) memcpy(colors + 3 * n_out, pt.col, 3);
        if (keys) keys[n_out] = pt.key;
        if (vis_counts) vis_counts[n_out] = (uint8_t)pt.vis.size();
        if (vis)
          for (uint32_t t = 0; t < vis_stride; ++t) vis[n_out * vis_stride + t] = t < pt.vis.size() ? pt.vis[t] : 0;
      }
      n_out++;
    }
  *count = n_out;
  if (residual_count) *residual_count = out2.size();
  return n_out <= capacity ? PS_OK : PS_EINVAL;
}

// ---- neighbour views and depth ranges from sparse tracks (crates/dense/src/neighbors.rs:44-186) ----------------
// DenseView::center (crates/dense/src/scene.rs:82-89): -(Rᵀ t).
static void nb_center(const ps_sparse_view& v, double c[3]) {
  for (int j = 0; j < 3; ++j) c[j] = -(v.r[0 * 3 + j] * v.t[0] + v.r[1 * 3 + j] * v.t[1] + v.r[2 * 3 + j] * v.t[2]);
}
// quantile_sorted (crates/dense/src/math.rs:126-135): linear interpolation between the order statistics around
// q·(n-1).
static double nb_quantile_sorted(const std::vector<double>& v, double q) {
  if (v.empty()) return 0.0;
  const double pos = q * (double)(v.size() - 1);
  const size_t lo = (size_t)std::floor(pos);
  const size_t hi = std::min(lo + 1, v.size() - 1);
  const double f = pos - (double)lo;
  return v[lo] + (v[hi] - v[lo]) * f;
}
// f64::powi as lowered for a run-time exponent: square-and-multiply over the exponent's bits, lowest bit first.
static double nb_powi(double a, int b) {
  const bool recip = b < 0;
  double r = 1.0;
  for (;;) {
    if (b & 1) r *= a;
    b /= 2;
    if (b == 0) break;
    a *= a;
  }
  return recip ? 1.0 / r : r;
}

void oracle_neighbor_params_default(ps_neighbor_params* out) {
  out->num_views = 10;
  out->direction_bins = 8;
  out->min_triangulation_angle_deg = 1.0;
  out->diversity_decay = 1.0;
}

int oracle_select_neighbors(const ps_sparse_view* views, uint32_t nv, const double* xyz, const uint32_t* toff,
                            const uint32_t* tview, uint64_t np, const ps_neighbor_params* prm, uint32_t* sources,
                            uint32_t* num_sources, double* depth_range, uint8_t* has_range, uint32_t* pair_count,
                            double* pair_angle75) {
  if (!views || !nv || !prm || !prm->num_views || !sources || !num_sources || (np && (!xyz || !toff || !tview)))
    return PS_EINVAL;
  for (uint64_t i = 0; i < np; ++i)
    for (uint32_t k = toff[i]; k < toff[i + 1]; ++k)
      if (tview[k] >= nv) return PS_EINVAL;
  std::vector<std::array<double, 3>> centers(nv);
  for (uint32_t v = 0; v < nv; ++v) nb_center(views[v], centers[v].data());
  // PairStats::new (neighbors.rs:47-76): every pair of distinct entries of a track, counted and its triangulation
  // angle min(a, pi - a) recorded in binary32
  const size_t nn = (size_t)nv * nv;
  std::vector<uint32_t> cnt(nn, 0);
  std::vector<std::vector<float>> angs(nn);
  for (uint64_t i = 0; i < np; ++i) {
    const double* x = xyz + 3 * i;
    for (uint32_t ii = toff[i]; ii < toff[i + 1]; ++ii)
      for (uint32_t jj = toff[i]; jj < ii; ++jj) {
        const uint32_t a = tview[ii], b = tview[jj];
        if (a == b) continue;
        const double* ca = centers[a].data();
        const double* cb = centers[b].data();
        const double u[3] = {ca[0] - x[0], ca[1] - x[1], ca[2] - x[2]};
        const double w[3] = {cb[0] - x[0], cb[1] - x[1], cb[2] - x[2]};
        const double nu = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        const double nw = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        double ang = 0.0;
        if (!(nu == 0.0 || nw == 0.0)) {
          double c = (u[0] * w[0] + u[1] * w[1] + u[2] * w[2]) / (nu * nw);
          if (c < -1.0) c = -1.0;
          else if (c > 1.0) c = 1.0;
          const double t = std::acos(c);
          ang = std::fmin(t, M_PI - t);
        }
        const size_t key = (size_t)std::min(a, b) * nv + std::max(a, b);
        cnt[key]++;
        angs[key].push_back((float)ang);
      }
  }
  std::vector<double> q75(nn, 0.0);
  for (size_t k = 0; k < nn; ++k) {
    if (!cnt[k]) continue;
    std::vector<double> a(angs[k].begin(), angs[k].end());
    std::sort(a.begin(), a.end());
    q75[k] = nb_quantile_sorted(a, 0.75);
  }
  if (pair_count) memcpy(pair_count, cnt.data(), nn * sizeof(uint32_t));
  if (pair_angle75) memcpy(pair_angle75, q75.data(), nn * sizeof(double));
  // select (neighbors.rs:82-101) with the angle in radians (f64::to_radians: deg · (pi/180)), and select_diverse
  // (neighbors.rs:108-150) when the decay is below 1 (densify.rs:224-240)
  const double min_angle = prm->min_triangulation_angle_deg * (M_PI / 180.0);
  const uint32_t maxn = prm->num_views;
  const bool diverse = prm->diversity_decay < 1.0;
  const size_t bins = std::max<uint32_t>(prm->direction_bins, 1);
  for (uint32_t r = 0; r < nv; ++r) {
    std::vector<std::pair<uint32_t, uint32_t>> cands;  // (count, view)
    for (uint32_t o = 0; o < nv; ++o) {
      if (o == r) continue;
      const size_t key = (size_t)std::min(r, o) * nv + std::max(r, o);
      if (!cnt[key]) continue;
      if (min_angle > 0.0 && q75[key] < min_angle) continue;
      cands.push_back({cnt[key], o});
    }
    std::sort(cands.begin(), cands.end(), [](const std::pair<uint32_t, uint32_t>& x, const std::pair<uint32_t, uint32_t>& y) {
      return x.first != y.first ? x.first > y.first : x.second < y.second;
    });
    std::vector<uint32_t> out;
    if (!diverse) {
      for (size_t i = 0; i < cands.size() && out.size() < maxn; ++i) out.push_back(cands[i].second);
    } else {
      const ps_sparse_view& vr = views[r];
      const double* cr = centers[r].data();
      std::vector<size_t> bin(cands.size());
      for (size_t i = 0; i < cands.size(); ++i) {
        const double* co = centers[cands[i].second].data();
        const double d[3] = {co[0] - cr[0], co[1] - cr[1], co[2] - cr[2]};
        double b[3];
        for (int k = 0; k < 3; ++k) b[k] = vr.r[k * 3 + 0] * d[0] + vr.r[k * 3 + 1] * d[1] + vr.r[k * 3 + 2] * d[2];
        const double lat = std::sqrt(b[0] * b[0] + b[1] * b[1]);
        if (lat < 0.3 * std::fabs(b[2])) {
          bin[i] = bins;
        } else {
          const double a = std::atan2(b[1], b[0]) + M_PI;
          bin[i] = std::min((size_t)(a / (2.0 * M_PI) * (double)bins), bins - 1);
        }
      }
      std::vector<int> used(bins + 1, 0);
      std::vector<char> taken(cands.size(), 0);
      while (out.size() < maxn) {
        bool any = false;
        double bs = 0.0;
        size_t bi = 0;
        for (size_t i = 0; i < cands.size(); ++i) {
          if (taken[i]) continue;
          const double sc = (double)cands[i].first * nb_powi(prm->diversity_decay, used[bin[i]]);
          if (!any || sc > bs) {
            any = true;
            bs = sc;
            bi = i;
          }
        }
        if (!any) break;
        taken[bi] = 1;
        used[bin[bi]]++;
        out.push_back(cands[bi].second);
      }
    }
    num_sources[r] = (uint32_t)out.size();
    for (uint32_t k = 0; k < maxn; ++k) sources[(size_t)r * maxn + k] = k < out.size() ? out[k] : UINT32_MAX;
  }
  // depth_ranges / depth_range_of (neighbors.rs:160-186): positive depths of every observation (repeats included),
  // the 1 % and 99 % order statistics (no interpolation) times 0.75 and 1.25
  std::vector<std::vector<double>> lists(nv);
  for (uint64_t i = 0; i < np; ++i) {
    const double* x = xyz + 3 * i;
    for (uint32_t k = toff[i]; k < toff[i + 1]; ++k) {
      const ps_sparse_view& v = views[tview[k]];
      const double d = v.r[6] * x[0] + v.r[7] * x[1] + v.r[8] * x[2] + v.t[2];
      if (d > 0.0) lists[tview[k]].push_back(d);
    }
  }
  for (uint32_t v = 0; v < nv; ++v) {
    std::vector<double>& l = lists[v];
    if (has_range) has_range[v] = l.empty() ? 0 : 1;
    if (!depth_range) continue;
    if (l.empty()) {
      depth_range[2 * v] = depth_range[2 * v + 1] = 0.0;
      continue;
    }
    std::sort(l.begin(), l.end());
    const size_t n = l.size();
    const double lo = l[std::min((size_t)std::floor((double)n * 0.01), n - 1)];
    const double hi = l[std::min((size_t)std::floor((double)n * 0.99), n - 1)];
    depth_range[2 * v] = 0.75 * lo;
    depth_range[2 * v + 1] = 1.25 * hi;
  }
  return PS_OK;
}

// filter_visibility (crates/dense/src/visibility.rs:106-151) on a bare cloud: keep[i] = 0 for the removed points;
// returns their number (0 when the filter is off: check_views, min_violations and tau must all be positive).
int64_t oracle_filter_visibility(uint32_t nviews, const ps_fusion_view* cams, const uint32_t* widths,
                                 const uint32_t* heights, const float* const* depth, const uint8_t* used,
                                 const float* positions, const uint8_t* vis_counts, const uint16_t* vis,
                                 uint32_t vis_stride, uint64_t n, uint32_t check_views, uint32_t min_violations,
                                 double tau, uint8_t* keep) {
  if (!cams || !widths || !heights || !depth || !used || (n && (!positions || !vis_counts || !vis || !keep)))
    return -1;
  std::vector<FCam> fc(nviews);
  for (uint32_t v = 0; v < nviews; ++v) {
    memcpy(fc[v].k, cams[v].k, sizeof fc[v].k);
    memcpy(fc[v].r, cams[v].r, sizeof fc[v].r);
    memcpy(fc[v].t, cams[v].t, sizeof fc[v].t);
    fc[v].w = (int)widths[v];
    fc[v].h = (int)heights[v];
  }
  const bool on = check_views > 0 && tau > 0.0 && min_violations > 0;
  int64_t removed = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const bool out = on && visibility_violated(positions + 3 * i, vis + i * vis_stride,
                                               std::min<uint32_t>(vis_counts[i], vis_stride), nviews, cams, fc, depth,
                                               used, check_views, min_violations, tau);
    keep[i] = out ? 0 : 1;
    removed += out;
  }
  return removed;
}

// smooth_along_normals on a bare cloud (positions updated in place); returns the median absolute displacement of the
// last pass, as the reference does.
double oracle_smooth(float* positions, const float* normals, uint64_t n, double gsd, uint32_t iterations,
                     double radius_gsd, double sigma_range_gsd, double normal_deg, int threads) {
  if ((!positions || !normals) && n) return -1.0;
  set_threads(threads);
  std::vector<float*> ppos(n);
  std::vector<const float*> pnrm(n);
  for (uint64_t i = 0; i < n; ++i) {
    ppos[i] = positions + 3 * i;
    pnrm[i] = normals + 3 * i;
  }
  return smooth_points(ppos, pnrm, gsd, iterations, radius_gsd, sigma_range_gsd, normal_deg);
}

// ---- score fusion (crates/dense/src/fusion_score.rs:196-435) -------------------------------------------------
// Candidates per reference pixel (view_candidates, fusion_score.rs:196-303) in (view, pixel) order; with mark_used the
// greedy choice in priority order (score descending, then view and pixel ascending): a candidate is adopted when none
// of its pixels (its own and its agreeing pixels) was taken by an adopted candidate before it, which is the result the
// reference's claim rounds reach (fusion_score.rs:352-414).  The exponentials and the arc cosine are ps_exp64 /
// ps_acos64, as in the engine.
int oracle_fuse_scored(uint32_t nviews, const ps_fusion_view* cams, const uint32_t* widths, const uint32_t* heights,
                       const float* const* depth, const float* const* normal, const float* const* cost,
                       const float* const* img, const uint8_t* used, const ps_score_fusion_params* p,
                       const ps_fusion_params* post, int threads, uint64_t capacity, float* positions, float* normals,
                       uint8_t* colors, uint64_t* keys, uint8_t* vis_counts, uint16_t* vis, uint32_t vis_stride,
                       uint64_t* count, uint64_t* visibility_removed) {
  if (!cams || !widths || !heights || !depth || !normal || !cost || !img || !used || !p || !count) return PS_EINVAL;
  set_threads(threads);
  std::vector<FCam> fc(nviews);
  std::vector<std::array<double, 3>> ctr(nviews);
  for (uint32_t v = 0; v < nviews; ++v) {
    memcpy(fc[v].k, cams[v].k, sizeof fc[v].k);
    memcpy(fc[v].r, cams[v].r, sizeof fc[v].r);
    memcpy(fc[v].t, cams[v].t, sizeof fc[v].t);
    fc[v].baseline = cams[v].baseline;
    fc[v].w = (int)widths[v];
    fc[v].h = (int)heights[v];
    for (int j = 0; j < 3; ++j)
      ctr[v][j] = -(fc[v].r[0 * 3 + j] * fc[v].t[0] + fc[v].r[1 * 3 + j] * fc[v].t[1] + fc[v].r[2 * 3 + j] * fc[v].t[2]);
  }
  std::vector<std::vector<int>> ovs(nviews);
  for (uint32_t v = 0; v < nviews; ++v) {
    if (!used[v]) continue;
    for (uint32_t j = 0; j < cams[v].num_overlap && ovs[v].size() < p->num_neighbors; ++j) {
      const uint32_t o = cams[v].overlap[j];
      if (o != v && o < nviews && used[o]) ovs[v].push_back((int)o);
    }
  }
  const double cos_n = std::cos(ps_to_radians_f64(p->normal_error_deg));
  const double k_e = 1.0 / (2.0 * p->sigma_e_px * p->sigma_e_px);
  const double st = ps_to_radians_f64(p->sigma_theta_deg);
  const double k_t = 1.0 / (2.0 * st * st);
  auto conf = [&](int v, size_t pix) { return std::min(std::max(1.0 - (double)cost[v][pix], 0.0), 1.0); };
  auto ivar = [&](int v, size_t pix, double d) {
    if (!p->inverse_variance || !(fc[v].baseline > 0.0)) return 1.0;
    const double spx = p->sigma_px0 + p->sigma_px_slope * (double)std::min(std::max(cost[v][pix], 0.0f), 2.0f);
    const double sd = d * d * spx / (fc[v].k[0] * fc[v].baseline);
    return 1.0 / std::max(sd * sd, 1e-300);
  };
  struct SCand {
    uint32_t v, pix;
    float score;
    FPoint pt;
    std::vector<std::pair<int, int>> hits;
  };
  std::vector<SCand> cands;
  for (uint32_t v = 0; v < nviews; ++v) {
    if (!used[v]) continue;
    const FCam& cv = fc[v];
    std::vector<std::vector<SCand>> rows(cv.h);
#pragma omp parallel for schedule(dynamic, 4)
    for (int row = 0; row < cv.h; ++row) {
      for (int col = 0; col < cv.w; ++col) {
        const size_t pix = (size_t)row * cv.w + col;
        const double d = (double)depth[v][pix];
        if (!(d > 0.0)) continue;  // NaN depths are invalid too (the reference's casts of NaN are undefined)
        double x[3], nw[3];
        f_backproject(cv, (double)col, (double)row, d, x);
        f_normal(cv, normal[v] + 3 * pix, nw);
        const double rr[3] = {x[0] - ctr[v][0], x[1] - ctr[v][1], x[2] - ctr[v][2]};
        const double l_ref = std::sqrt(rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2]);
        const double s_ref = conf((int)v, pix);
        const double w0 = s_ref * ivar((int)v, pix, d);
        double sum_s = s_ref, sum_p = 0.0, sw = w0;
        double sx[3] = {x[0] * w0, x[1] * w0, x[2] * w0};
        double sn[3] = {nw[0] * w0, nw[1] * w0, nw[2] * w0};
        const double c0 = f_gray(img[v], cv, col, row);
        double sc[3] = {c0 * w0, c0 * w0, c0 * w0};
        std::vector<std::pair<int, int>> hits;
        for (int j : ovs[v]) {
          const FCam& oc = fc[j];
          double u, vv, z;
          if (!f_project(oc, x, &u, &vv, &z)) continue;
          const double cu = std::floor(u + 0.5), rv = std::floor(vv + 0.5);
          if (cu < 0.0 || rv < 0.0 || cu >= (double)oc.w || rv >= (double)oc.h) continue;
          const size_t opix = (size_t)rv * oc.w + (size_t)cu;
          const double od = (double)depth[j][opix];
          if (od <= 0.0) continue;
          const double cj = conf(j, opix);
          if (std::fabs(z - od) / od > p->depth_error) {
            if (z < od * (1.0 - p->depth_error)) sum_p += cj;
            continue;
          }
          double no[3];
          f_normal(oc, normal[j] + 3 * opix, no);
          if (no[0] * nw[0] + no[1] * nw[1] + no[2] * nw[2] < cos_n) continue;
          double xo[3];
          f_backproject(oc, cu, rv, od, xo);
          double bu, bv, bz;
          if (!f_project(cv, xo, &bu, &bv, &bz)) continue;
          const double eu = bu - (double)col, ev = bv - (double)row;
          const double e2 = eu * eu + ev * ev;
          const double rj[3] = {x[0] - ctr[j][0], x[1] - ctr[j][1], x[2] - ctr[j][2]};
          double cos_t = (rr[0] * rj[0] + rr[1] * rj[1] + rr[2] * rj[2]) /
                         (l_ref * std::sqrt(rj[0] * rj[0] + rj[1] * rj[1] + rj[2] * rj[2]));
          cos_t = std::min(std::max(cos_t, -1.0), 1.0);
          const double th = ps_acos64(cos_t);
          const double sj = cj * ps_exp64(-e2 * k_e) * (1.0 - ps_exp64(-th * th * k_t));
          sum_s += sj;
          if (sj <= 0.0) continue;
          const double wo = sj * ivar(j, opix, od);
          const double co = f_gray(img[j], oc, (int)cu, (int)rv);
          sw += wo;
          for (int k = 0; k < 3; ++k) {
            sx[k] += wo * xo[k];
            sn[k] += wo * no[k];
            sc[k] += wo * co;
          }
          hits.push_back({j, (int)opix});
        }
        const double score = sum_s - p->lambda * sum_p;
        if (score < p->tau || sw <= 0.0 || !std::isfinite(sw)) continue;
        const double l = std::sqrt(sn[0] * sn[0] + sn[1] * sn[1] + sn[2] * sn[2]);
        if (l < 1.1920928955078125e-07) continue;
        SCand c;
        c.v = v;
        c.pix = (uint32_t)pix;
        c.score = (float)score;
        for (int k = 0; k < 3; ++k) {
          c.pt.pos[k] = (float)(sx[k] / sw);
          c.pt.nrm[k] = (float)(sn[k] / l);
          c.pt.col[k] = (uint8_t)std::min(std::max(std::round(sc[k] / sw), 0.0), 255.0);
        }
        c.pt.key = ((uint64_t)cams[v].image_id << 32) | ((uint64_t)(row & 0xffff) << 16) | (uint64_t)(col & 0xffff);
        c.pt.vis.assign(1, (uint16_t)v);
        for (auto& hq : hits) c.pt.vis.push_back((uint16_t)hq.first);
        std::sort(c.pt.vis.begin(), c.pt.vis.end());
        c.pt.vis.erase(std::unique(c.pt.vis.begin(), c.pt.vis.end()), c.pt.vis.end());
        c.hits = std::move(hits);
        rows[row].push_back(std::move(c));
      }
    }
    for (auto& r : rows)
      for (auto& c : r) cands.push_back(std::move(c));
  }
  std::vector<char> accepted(cands.size(), p->mark_used ? 0 : 1);
  if (p->mark_used && !cands.empty()) {
    std::vector<size_t> order(cands.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;  // (view, pixel) order already
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
      const uint32_t ka = ps_f2u(cands[a].score), kb = ps_f2u(cands[b].score);
      const uint32_t oa = (ka & 0x80000000u) ? ~ka : (ka | 0x80000000u), ob = (kb & 0x80000000u) ? ~kb : (kb | 0x80000000u);
      return oa > ob;  // score descending in total order; ties keep (view, pixel) order
    });
    std::vector<std::vector<char>> taken(nviews);
    for (uint32_t v = 0; v < nviews; ++v)
      if (used[v]) taken[v].assign((size_t)fc[v].w * fc[v].h, 0);
    for (size_t g : order) {
      const SCand& c = cands[g];
      bool free = !taken[c.v][c.pix];
      for (auto& hq : c.hits) free = free && !taken[hq.first][hq.second];
      if (!free) continue;
      accepted[g] = 1;
      taken[c.v][c.pix] = 1;
      for (auto& hq : c.hits) taken[hq.first][hq.second] = 1;
    }
  }
  // fuse_depth_maps_with (crates/dense/src/densify.rs:535-556): the visibility filter, then the smoothing, on the
  // adopted points in their order, with the fusion's overlap lists and the scene GSD of the fused views
  uint64_t vis_removed = 0;
  if (post && post->visibility_check_views > 0 && post->visibility_tau > 0.0 && post->visibility_min_violations > 0)
    for (size_t g = 0; g < cands.size(); ++g) {
      if (!accepted[g]) continue;
      const FPoint& pt = cands[g].pt;
      if (visibility_violated(pt.pos, pt.vis.data(), pt.vis.size(), nviews, cams, fc, depth, used,
                              post->visibility_check_views, post->visibility_min_violations, post->visibility_tau)) {
        accepted[g] = 0;
        vis_removed++;
      }
    }
  if (visibility_removed) *visibility_removed = vis_removed;
  if (post && post->smooth_iterations > 0) {
    std::vector<float*> ppos;
    std::vector<const float*> pnrm;
    for (size_t g = 0; g < cands.size(); ++g)
      if (accepted[g]) {
        ppos.push_back(cands[g].pt.pos);
        pnrm.push_back(cands[g].pt.nrm);
      }
    smooth_points(ppos, pnrm, scene_gsd(nviews, fc, depth, used), post->smooth_iterations, post->smooth_radius_gsd,
                  post->smooth_sigma_range_gsd, post->smooth_normal_deg);
  }
  uint64_t n_out = 0;
  for (size_t g = 0; g < cands.size(); ++g) {
    if (!accepted[g]) continue;
    const FPoint& pt = cands[g].pt;
    if (n_out < capacity) {
      if (positions) memcpy(positions + 3 * n_out, pt.pos, 12);
      if (normals) memcpy(normals + 3 * n_out, pt.nrm, 12);
      if (colors) memcpy(colors + 3 * n_out, pt.col, 3);
      if (keys) keys[n_out] = pt.key;
      if (vis_counts) vis_counts[n_out] = (uint8_t)pt.vis.size();
      if (vis)
        for (uint32_t t = 0; t < vis_stride; ++t) vis[n_out * vis_stride + t] = t < pt.vis.size() ? pt.vis[t] : 0;
    }
    n_out++;
  }
  *count = n_out;
  return n_out <= capacity ? PS_OK : PS_EINVAL;
}

}  // extern "C"
