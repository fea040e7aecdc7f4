// Post-processing of resident depth maps: speckle removal and consistency fusion.
//
//   * Speckle removal restates remove_speckles (crates/dense/src/postproc.rs:77-129): 4-connected components of valid
//     pixels, two neighbours joined when |d_j - d_i| <= rel·min(d_i, d_j); a component smaller than
//     ceil(w·h·min_area_frac) whose lower median cost (sorted costs[len/2]) exceeds keep_cost is erased.  The
//     reference grows components by depth-first search from the first pixel in row-major order; the components of this
//     symmetric relation do not depend on the order, so the GPU labels them with a lock-free union-find (roots hook to
//     the smaller index, so each label is the component's first pixel) and finds the lower median of each small
//     component exactly by bisection over an order-preserving integer key of the f32 costs.
//   * Consistency fusion restates fuse_consistency with residual handling "none" (crates/dense/src/fusion.rs:219-459):
//     views in the caller's order, every reference pixel of a view evaluated independently in FP64 (projection,
//     back-projection, reprojection error, normal agreement, inverse-variance weighted means).  Within one view the
//     evaluation reads only marks that earlier views wrote and writes marks of other views, so one kernel launch per
//     view reproduces the reference's result exactly; points are appended in any order and carry the reference's
//     point key, so sorting by key restores the reference's order (views ascending, row-major within a view).
//
// This file is compiled with the parity flags (no contraction, IEEE division and square root): the FP64 operation
// sequence matches the CPU oracle's restatement operation by operation.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "ps_post.h"
#include "ps_fmath.h"

namespace ps_post {

// ------------------------------------------------------------------------------------------- speckles
__device__ __forceinline__ int item_of(const SpkArgs& A, int cta) {
  int lo = 0, hi = A.nitems - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (A.items[mid].tile0 <= cta) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct Px {
  int x, y, g;  // pixel and its slot index
  const SpkItem* it;
};

__device__ __forceinline__ bool spk_px(const SpkArgs& A, Px& p) {
  const int ii = item_of(A, blockIdx.x);
  const SpkItem& it = A.items[ii];
  const int tiles_x = (it.w + 31) / 32;
  const int tl = blockIdx.x - it.tile0;
  p.x = (tl % tiles_x) * 32 + threadIdx.x;
  p.y = (tl / tiles_x) * 8 + threadIdx.y;
  p.it = &it;
  if (p.x >= it.w || p.y >= it.h) return false;
  p.g = (int)(it.off + (long long)p.y * it.w + p.x);
  return true;
}

// Order-preserving key of an f32 (IEEE total order): keys compare like the floats (−0 before +0).
__device__ __forceinline__ unsigned fkey(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float funkey(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

__device__ __forceinline__ int find_root(const int* parent, int x) {
  int p;
  while ((p = __ldcg(parent + x)) != x) x = p;  // L2 reads: parents change during the union pass
  return x;
}

// Joins the components of a and b: the larger root is hooked under the smaller with a compare-and-swap; a failed swap
// means the root got a (smaller) parent meanwhile, so the loop continues from it.  Each retry strictly lowers `a`.
__device__ void unite(int* parent, int a, int b) {
  while (true) {
    a = find_root(parent, a);
    b = find_root(parent, b);
    if (a == b) return;
    if (a < b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicCAS(parent + a, a, b);
    if (old == a) return;
    a = old;
  }
}

__device__ __forceinline__ bool joined(float di, float dj, float rel) {
  return dj > 0.f && fabsf(dj - di) <= rel * fminf(di, dj);
}

__global__ void k_spk_init(SpkArgs A) {
  Px p;
  if (!spk_px(A, p)) return;
  A.parent[p.g] = A.plane[p.g].w > 0.f ? p.g : -1;
  A.size[p.g] = 0;
  A.cnt[p.g] = 0;
}

__global__ void k_spk_union(SpkArgs A) {
  Px p;
  if (!spk_px(A, p)) return;
  const float di = A.plane[p.g].w;
  if (!(di > 0.f)) return;
  if (p.x + 1 < p.it->w && joined(di, A.plane[p.g + 1].w, A.rel)) unite(A.parent, p.g, p.g + 1);
  if (p.y + 1 < p.it->h && joined(di, A.plane[p.g + p.it->w].w, A.rel)) unite(A.parent, p.g, p.g + p.it->w);
}

__global__ void k_spk_flatten(SpkArgs A) {
  Px p;
  if (!spk_px(A, p)) return;
  if (A.parent[p.g] < 0) return;
  const int r = find_root(A.parent, p.g);
  A.parent[p.g] = r;
  atomicAdd(A.size + r, 1);
}

// Small components: bisection state [lo, hi] over cost keys for the lower median (the (size/2)-th smallest key).
__global__ void k_spk_bisect_init(SpkArgs A) {
  Px p;
  if (!spk_px(A, p)) return;
  if (A.parent[p.g] != p.g || A.size[p.g] >= p.it->min_area) return;
  A.lo[p.g] = 0u;
  A.hi[p.g] = 0xFFFFFFFFu;
}

__global__ void k_spk_count(SpkArgs A) {
  Px p;
  if (!spk_px(A, p)) return;
  const int r = A.parent[p.g];
  if (r < 0 || A.size[r] >= p.it->min_area) return;
  const unsigned lo = A.lo[r], hi = A.hi[r];
  const unsigned mid = lo + (hi - lo) / 2u;
  if (fkey(A.cost[p.g]) <= mid) atomicAdd(A.cnt + r, 1u);
}

__global__ void k_spk_step(SpkArgs A) {
  Px p;
  if (!spk_px(A, p)) return;
  if (A.parent[p.g] != p.g || A.size[p.g] >= p.it->min_area) return;
  const unsigned lo = A.lo[p.g], hi = A.hi[p.g];
  const unsigned mid = lo + (hi - lo) / 2u;
  const unsigned k = (unsigned)A.size[p.g] / 2u;
  if (A.cnt[p.g] >= k + 1u) A.hi[p.g] = mid;
  else A.lo[p.g] = mid + 1u;
  A.cnt[p.g] = 0u;
}

__global__ void k_spk_erase(SpkArgs A) {
  Px p;
  if (!spk_px(A, p)) return;
  const int r = A.parent[p.g];
  if (r < 0 || A.size[r] >= p.it->min_area) return;
  if (funkey(A.lo[r]) > A.keep) {
    A.plane[p.g] = make_float4(0.f, 0.f, 0.f, 0.f);
    atomicAdd(A.removed, 1ull);
  }
}

__global__ void k_count_valid(SpkArgs A) {
  Px p;
  const bool ok = spk_px(A, p) && A.plane[p.g].w > 0.f;
  const unsigned m = __ballot_sync(0xffffffffu, ok);
  if (threadIdx.x == 0 && m) atomicAdd(A.valid, (unsigned long long)__popc(m));
}

cudaError_t launch_count_valid(const SpkArgs& A, int ntiles, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  k_count_valid<<<ntiles, dim3(32, 8), 0, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_speckles(const SpkArgs& A, int ntiles, cudaStream_t st, int* launches) {
  if (ntiles <= 0) return cudaSuccess;
  const dim3 b(32, 8);
  k_spk_init<<<ntiles, b, 0, st>>>(A);
  k_spk_union<<<ntiles, b, 0, st>>>(A);
  k_spk_flatten<<<ntiles, b, 0, st>>>(A);
  k_spk_bisect_init<<<ntiles, b, 0, st>>>(A);
  for (int i = 0; i < 32; ++i) {  // 32 halvings of the 2^32 key range leave lo == hi
    k_spk_count<<<ntiles, b, 0, st>>>(A);
    k_spk_step<<<ntiles, b, 0, st>>>(A);
  }
  k_spk_erase<<<ntiles, b, 0, st>>>(A);
  *launches += 5 + 64;
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------- fusion
struct Hit {
  int o, q;
};

// camera -> world of pixel (col, row) at depth d: X = Rᵀ (c - t), c = ((col-cx)/fx·d, (row-cy)/fy·d, d)
__device__ __forceinline__ void backproject(const FuseView& c, double col, double row, double d, double* X) {
  const double cc[3] = {(col - c.k[2]) / c.k[0] * d, (row - c.k[3]) / c.k[1] * d, d};
  const double p[3] = {cc[0] - c.t[0], cc[1] - c.t[1], cc[2] - c.t[2]};
  const double* r = c.r;
  X[0] = r[0] * p[0] + r[3] * p[1] + r[6] * p[2];
  X[1] = r[1] * p[0] + r[4] * p[1] + r[7] * p[2];
  X[2] = r[2] * p[0] + r[5] * p[1] + r[8] * p[2];
}

__device__ __forceinline__ bool project(const FuseView& c, const double* x, double* u, double* v, double* z) {
  const double* r = c.r;
  const double cz = r[6] * x[0] + r[7] * x[1] + r[8] * x[2] + c.t[2];
  if (cz <= 0.0) return false;
  const double cx = r[0] * x[0] + r[1] * x[1] + r[2] * x[2] + c.t[0];
  const double cy = r[3] * x[0] + r[4] * x[1] + r[5] * x[2] + c.t[1];
  *u = c.k[0] * cx / cz + c.k[2];
  *v = c.k[1] * cy / cz + c.k[3];
  *z = cz;
  return true;
}

__device__ __forceinline__ void normal_world(const FuseView& c, float4 q, double* n) {
  const double m[3] = {(double)q.x, (double)q.y, (double)q.z};
  const double* r = c.r;
  n[0] = r[0] * m[0] + r[3] * m[1] + r[6] * m[2];
  n[1] = r[1] * m[0] + r[4] * m[1] + r[7] * m[2];
  n[2] = r[2] * m[0] + r[5] * m[1] + r[8] * m[2];
}

// inv_var (crates/dense/src/fusion.rs:86-95): 1/σ_d² with σ_d = d²·σ_px/(f·b), σ_px = σ0 + slope·clamp(cost, 0, 2).
__device__ __forceinline__ double inv_var(const FuseArgs& A, const FuseView& c, double d, float cost) {
  if (!A.inverse_variance || !(c.baseline > 0.0)) return 1.0;
  const double spx = A.sigma0 + A.slope * (double)fminf(fmaxf(cost, 0.0f), 2.0f);
  const double sd = d * d * spx / (c.k[0] * c.baseline);
  return 1.0 / fmax(sd * sd, 1e-300);
}

// Gray u8 colour of an image plane value (the reference uses the view's colour image; these images are gray).
__device__ __forceinline__ double gray_u8(const FuseView& c, int col, int row) {
  const int x = min(col, c.w - 1), y = min(row, c.h - 1);
  const float v = c.img[(long long)y * c.pitch + x] * 255.0f;
  return (double)(unsigned char)fminf(fmaxf(rintf(v), 0.0f), 255.0f);
}

// The agreement check of one reference pixel (ConsCtx::evaluate, crates/dense/src/fusion.rs:390-460) under the
// tolerances of A: the weighted sums of the point and its agreeing (view, pixel) list; false when the normal sum
// vanishes.
struct FusePoint {
  double sx[3], sn[3], sc[3], m, l;
};
__device__ bool fuse_eval(const FuseArgs& A, const FuseView& cv, int col, int row, float4 q, Hit* hits, int& nh,
                          FusePoint& P) {
  const double d = (double)q.w;
  double x[3], nw[3];
  backproject(cv, (double)col, (double)row, d, x);
  normal_world(cv, q, nw);
  const double w0 = inv_var(A, cv, d, A.cost[cv.off + (long long)row * cv.w + col]);
  double sw = w0;
  for (int k = 0; k < 3; ++k) {
    P.sx[k] = x[k] * w0;
    P.sn[k] = nw[k] * w0;
  }
  const double c0 = gray_u8(cv, col, row);
  P.sc[0] = P.sc[1] = P.sc[2] = c0 * w0;
  nh = 0;
  for (int i = 0; i < cv.nov; ++i) {
    const int o = cv.ov[i];
    const FuseView& oc = A.views[o];
    double u, vv, z;
    if (!project(oc, x, &u, &vv, &z)) continue;
    const double cu = floor(u + 0.5), rv = floor(vv + 0.5);
    if (cu < 0.0 || rv < 0.0 || cu >= (double)oc.w || rv >= (double)oc.h) continue;
    const int opix = (int)rv * oc.w + (int)cu;
    const float4 oq = A.plane[oc.off + opix];
    const double od = (double)oq.w;
    if (od <= 0.0 || fabs(z - od) / od > A.depth_tol) continue;
    double xo[3];
    backproject(oc, cu, rv, od, xo);
    double bu, bv, bz;
    if (!project(cv, xo, &bu, &bv, &bz)) continue;
    const double eu = bu - (double)col, ev = bv - (double)row;
    if (eu * eu + ev * ev > A.r2) continue;
    double no[3];
    normal_world(oc, oq, no);
    if (no[0] * nw[0] + no[1] * nw[1] + no[2] * nw[2] < A.cos_n) continue;
    const double co = gray_u8(oc, (int)cu, (int)rv);
    const double wo = inv_var(A, oc, od, A.cost[oc.off + opix]);
    sw += wo;
    for (int k = 0; k < 3; ++k) {
      P.sx[k] += wo * xo[k];
      P.sn[k] += wo * no[k];
      P.sc[k] += wo * co;
    }
    hits[nh].o = o;
    hits[nh].q = opix;
    nh++;
  }
  P.m = sw;
  P.l = sqrt(P.sn[0] * P.sn[0] + P.sn[1] * P.sn[1] + P.sn[2] * P.sn[2]);
  return !(P.l < 1.1920928955078125e-07);  // f32::EPSILON
}

// The sorted, de-duplicated {v} ∪ hit views into vis; returns their number.
__device__ int write_vis(unsigned short* vis, int v, const Hit* hits, int nh) {
  int nv = 0;
  vis[nv++] = (unsigned short)v;
  for (int i = 0; i < nh; ++i) {
    const unsigned short o = (unsigned short)hits[i].o;
    int j = nv;
    bool dup = false;
    for (int k = 0; k < nv; ++k) dup = dup || vis[k] == o;
    if (dup) continue;
    while (j > 0 && vis[j - 1] > o) {
      vis[j] = vis[j - 1];
      --j;
    }
    vis[j] = o;
    nv++;
  }
  return nv;
}

// Writes one fused point (its slot from the shared counter): mean position, normalised normal, rounded colour, key
// and the sorted, de-duplicated {v} ∪ hit views.
__device__ void fuse_emit(const FuseArgs& A, const FuseView& cv, int v, int col, int row, const FusePoint& P,
                          const Hit* hits, int nh) {
  const unsigned long long slot = atomicAdd(A.count, 1ull);
  if (slot >= A.capacity) return;  // cannot happen: capacity = valid pixels of the fused views
  for (int k = 0; k < 3; ++k) {
    A.pos[3 * slot + k] = (float)(P.sx[k] / P.m);
    A.nrm[3 * slot + k] = (float)(P.sn[k] / P.l);
    A.col[3 * slot + k] = (unsigned char)round(P.sc[k] / P.m);
  }
  A.key[slot] = ((unsigned long long)cv.image_id << 32) | ((unsigned long long)(row & 0xffff) << 16) |
                (unsigned long long)(col & 0xffff);
  A.nvis[slot] = (unsigned char)write_vis(A.vis + slot * A.vis_stride, v, hits, nh);
}

// First pass (fusion.rs:243-333) of view A.v: one thread per reference pixel.
__global__ void __launch_bounds__(256) k_fuse(FuseArgs A) {
  const FuseView& cv = A.views[A.v];
  const int col = blockIdx.x * 32 + threadIdx.x, row = blockIdx.y * 8 + threadIdx.y;
  if (col >= cv.w || row >= cv.h) return;
  const long long pix = (long long)row * cv.w + col;
  const float4 q = A.plane[cv.off + pix];
  if (!(q.w > 0.0f)) return;
  if (A.mark_used && A.marks[cv.off + pix] != 0) return;
  Hit hits[PS_FUSE_MAX_OVERLAP];
  int nh;
  FusePoint P;
  const bool okp = fuse_eval(A, cv, col, row, q, hits, nh, P);
  if (nh < A.min_views || !okp) return;
  if (A.mark_used) {
    for (int i = 0; i < nh; ++i) {
      const FuseView& oc = A.views[hits[i].o];
      if (A.mark_radius == 0) {
        A.marks[oc.off + hits[i].q] = 1;
        continue;
      }
      // marks within the radius whose depth agrees with the hit (crates/dense/src/fusion.rs:363-388)
      const int cx0 = hits[i].q % oc.w, cy0 = hits[i].q / oc.w, r = A.mark_radius;
      const double d0 = (double)A.plane[oc.off + hits[i].q].w;
      for (int yy = max(cy0 - r, 0); yy <= min(cy0 + r, oc.h - 1); ++yy)
        for (int xx = max(cx0 - r, 0); xx <= min(cx0 + r, oc.w - 1); ++xx) {
          const long long qq = (long long)yy * oc.w + xx;
          const double dq = (double)A.plane[oc.off + qq].w;
          if (dq > 0.0 && fabs(dq - d0) <= A.depth_tol * d0) A.marks[oc.off + qq] = 1;
        }
    }
  }
  if (A.consumed) {
    A.consumed[cv.off + pix] = 1;
    for (int i = 0; i < nh; ++i) A.consumed[A.views[hits[i].o].off + hits[i].q] = 1;
  }
  fuse_emit(A, cv, A.v, col, row, P, hits, nh);
}

// ---- second pass of leftover pixels (fusion.rs:540-627) ------------------------------------------------------
__device__ __forceinline__ unsigned long long grid_mix(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
// Slot key of a cell (never 0, the empty marker).  Different cells may share a key; the distance test keeps the
// result exact, since every point within the cell size lies in one of the 27 cells around.
__device__ __forceinline__ unsigned long long grid_key(long long cx, long long cy, long long cz) {
  const unsigned long long h =
      grid_mix((unsigned long long)cx ^ grid_mix((unsigned long long)cy ^ grid_mix((unsigned long long)cz)));
  return h ? h : 1ull;
}
__device__ __forceinline__ long long grid_cell(float x, double cell) { return (long long)floor((double)x / cell); }

__global__ void __launch_bounds__(256) k_grid_insert(const float* pos, unsigned n, double cell,
                                                     unsigned long long* keys, unsigned* heads, unsigned* next,
                                                     unsigned cap, int* overflow) {
  const unsigned i = blockIdx.x * 256u + threadIdx.x;
  if (i >= n) return;
  const unsigned long long key = grid_key(grid_cell(pos[3 * i], cell), grid_cell(pos[3 * i + 1], cell),
                                          grid_cell(pos[3 * i + 2], cell));
  unsigned slot = (unsigned)(key & (cap - 1));
  for (unsigned t = 0; t < cap; ++t) {
    const unsigned long long prev = atomicCAS(&keys[slot], 0ull, key);
    if (prev == 0ull || prev == key) {
      next[i] = atomicExch(&heads[slot], i);
      return;
    }
    slot = (slot + 1u) & (cap - 1u);
  }
  atomicExch(overflow, 1);  // cannot happen: the table is at most half full
}

// GridIndex::any_within (fusion.rs:514-536): is a first-pass point within the cell size of x (binary64 distance)?
__device__ bool grid_any_within(const FuseArgs& A, const float* x) {
  const long long c0 = grid_cell(x[0], A.gcell), c1 = grid_cell(x[1], A.gcell), c2 = grid_cell(x[2], A.gcell);
  const double rr = A.gcell * A.gcell;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const unsigned long long key = grid_key(c0 + dx, c1 + dy, c2 + dz);
        unsigned slot = (unsigned)(key & (A.gcap - 1));
        for (unsigned t = 0; t < A.gcap; ++t) {
          const unsigned long long k = A.gkeys[slot];
          if (k == 0ull) break;
          if (k == key) {
            unsigned i = A.gheads[slot];
            for (unsigned u = 0; u < A.gpoints && i != 0xffffffffu; ++u, i = A.gnext[i]) {
              const double t0 = (double)A.pos[3 * i] - (double)x[0];
              const double t1 = (double)A.pos[3 * i + 1] - (double)x[1];
              const double t2 = (double)A.pos[3 * i + 2] - (double)x[2];
              if ((t0 * t0 + t1 * t1) + t2 * t2 <= rr) return true;
            }
            break;
          }
          slot = (slot + 1u) & (A.gcap - 1u);
        }
      }
  return false;
}

// Stage 1: a leftover pixel (valid, not consumed by the first pass) that agrees with residual_min_views views under
// the second-pass tolerances and is not within the minimum distance of a first-pass point claims its own pixel and
// its agreeing pixels with its candidate number (atomic minimum).  Stage 2: a candidate that owns its reference pixel
// is emitted (only its own candidate writes its number there, so the test also says it was a candidate); its point
// is evaluated again with the same inputs.
__global__ void __launch_bounds__(256) k_fuse_second(FuseArgs A, int stage) {
  const FuseView& cv = A.views[A.v];
  const int col = blockIdx.x * 32 + threadIdx.x, row = blockIdx.y * 8 + threadIdx.y;
  if (col >= cv.w || row >= cv.h) return;
  const long long pix = (long long)row * cv.w + col;
  const unsigned id = cv.idbase + (unsigned)pix;
  if (stage == 2 && A.owner[cv.off + pix] != id) return;
  const float4 q = A.plane[cv.off + pix];
  if (!(q.w > 0.0f) || A.consumed[cv.off + pix] != 0) return;
  Hit hits[PS_FUSE_MAX_OVERLAP];
  int nh;
  FusePoint P;
  if (!fuse_eval(A, cv, col, row, q, hits, nh, P)) return;
  if (nh < A.min_views) return;
  if (stage == 1) {
    if (A.gcap) {
      const float x[3] = {(float)(P.sx[0] / P.m), (float)(P.sx[1] / P.m), (float)(P.sx[2] / P.m)};
      if (grid_any_within(A, x)) return;
    }
    atomicMin(&A.owner[cv.off + pix], id);
    for (int i = 0; i < nh; ++i) atomicMin(&A.owner[A.views[hits[i].o].off + hits[i].q], id);
    return;
  }
  fuse_emit(A, cv, A.v, col, row, P, hits, nh);
}

// ---- score fusion (crates/dense/src/fusion_score.rs:196-435) -------------------------------------------------
// Comparisons spelled as the CPU restatement's std::min / std::max, so that NaN inputs take the same branch there.
__device__ __forceinline__ double sc_clamp(double x, double lo, double hi) {
  x = x < lo ? lo : x;
  return hi < x ? hi : x;
}
// camera centre -Rᵀ t (DenseView::center, crates/dense/src/scene.rs:82-89)
__device__ __forceinline__ void sc_centre(const FuseView& c, double* o) {
  for (int j = 0; j < 3; ++j) o[j] = -(c.r[0 * 3 + j] * c.t[0] + c.r[1 * 3 + j] * c.t[1] + c.r[2 * 3 + j] * c.t[2]);
}
// inv_var (fusion_score.rs:161-171)
__device__ __forceinline__ double sc_inv_var(const ScoreArgs& A, const FuseView& c, double d, float cost) {
  if (!A.inverse_variance || !(c.baseline > 0.0)) return 1.0;
  float cc = cost < 0.0f ? 0.0f : cost;
  cc = 2.0f < cc ? 2.0f : cc;
  const double spx = A.sigma0 + A.slope * (double)cc;
  const double sd = d * d * spx / (c.k[0] * c.baseline);
  const double v = sd * sd;
  return 1.0 / (v < 1e-300 ? 1e-300 : v);
}
// IEEE total order of binary32 as an unsigned key (f32::total_cmp)
__device__ __forceinline__ unsigned sc_total_key(float f) {
  const unsigned k = __float_as_uint(f);
  return (k & 0x80000000u) ? ~k : (k | 0x80000000u);
}

// view_candidates (fusion_score.rs:196-303): one thread per reference pixel of view A.v.  The reference walks its
// pixels in order; here each candidate takes the next free record and its candidate number restores the order.
__global__ void __launch_bounds__(256) k_score(const ScoreArgs A) {
  const FuseView& cv = A.views[A.v];
  const int col = blockIdx.x * 32 + threadIdx.x, row = blockIdx.y * 8 + threadIdx.y;
  if (col >= cv.w || row >= cv.h) return;
  const long long pix = (long long)row * cv.w + col;
  const float4 q = A.plane[cv.off + pix];
  const double d = (double)q.w;
  if (!(d > 0.0)) return;
  double x[3], nw[3], cr[3];
  backproject(cv, (double)col, (double)row, d, x);
  normal_world(cv, q, nw);
  sc_centre(cv, cr);
  const double rr[3] = {x[0] - cr[0], x[1] - cr[1], x[2] - cr[2]};
  const double l_ref = sqrt(rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2]);
  const float cost0 = A.cost[cv.off + pix];
  const double s_ref = sc_clamp(1.0 - (double)cost0, 0.0, 1.0);
  const double w0 = s_ref * sc_inv_var(A, cv, d, cost0);
  double sum_s = s_ref, sum_p = 0.0, sw = w0, sx[3], sn[3], sc[3];
  for (int k = 0; k < 3; ++k) {
    sx[k] = x[k] * w0;
    sn[k] = nw[k] * w0;
  }
  const double c0 = gray_u8(cv, col, row);
  sc[0] = sc[1] = sc[2] = c0 * w0;
  Hit hits[PS_FUSE_MAX_OVERLAP];
  int nh = 0;
  for (int i = 0; i < cv.nov; ++i) {
    const int j = cv.ov[i];
    const FuseView& oc = A.views[j];
    double u, vv, z;
    if (!project(oc, x, &u, &vv, &z)) continue;
    const double cu = floor(u + 0.5), rv = floor(vv + 0.5);
    if (cu < 0.0 || rv < 0.0 || cu >= (double)oc.w || rv >= (double)oc.h) continue;
    const int opix = (int)rv * oc.w + (int)cu;
    const float4 oq = A.plane[oc.off + opix];
    const double od = (double)oq.w;
    if (od <= 0.0) continue;
    const float ocost = A.cost[oc.off + opix];
    const double cj = sc_clamp(1.0 - (double)ocost, 0.0, 1.0);
    if (fabs(z - od) / od > A.depth_tol) {
      if (z < od * (1.0 - A.depth_tol)) sum_p += cj;  // free-space violation
      continue;
    }
    double no[3];
    normal_world(oc, oq, no);
    if (no[0] * nw[0] + no[1] * nw[1] + no[2] * nw[2] < A.cos_n) continue;
    double xo[3];
    backproject(oc, cu, rv, od, xo);
    double bu, bv, bz;
    if (!project(cv, xo, &bu, &bv, &bz)) continue;
    const double eu = bu - (double)col, ev = bv - (double)row;
    const double e2 = eu * eu + ev * ev;
    double cj3[3];
    sc_centre(oc, cj3);
    const double rj[3] = {x[0] - cj3[0], x[1] - cj3[1], x[2] - cj3[2]};
    const double cos_t = sc_clamp((rr[0] * rj[0] + rr[1] * rj[1] + rr[2] * rj[2]) /
                                      (l_ref * sqrt(rj[0] * rj[0] + rj[1] * rj[1] + rj[2] * rj[2])),
                                  -1.0, 1.0);
    const double th = ps_acos64(cos_t);
    const double sj = cj * ps_exp64(-e2 * A.k_e) * (1.0 - ps_exp64(-th * th * A.k_t));
    sum_s += sj;
    if (sj <= 0.0) continue;
    const double wo = sj * sc_inv_var(A, oc, od, ocost);
    const double co = gray_u8(oc, (int)cu, (int)rv);
    sw += wo;
    for (int k = 0; k < 3; ++k) {
      sx[k] += wo * xo[k];
      sn[k] += wo * no[k];
      sc[k] += wo * co;
    }
    hits[nh].o = j;
    hits[nh].q = opix;
    nh++;
  }
  const double score = sum_s - A.lambda * sum_p;
  if (score < A.tau || sw <= 0.0 || !isfinite(sw)) return;
  const double l = sqrt(sn[0] * sn[0] + sn[1] * sn[1] + sn[2] * sn[2]);
  if (l < 1.1920928955078125e-07) return;  // f32::EPSILON
  const unsigned long long c = atomicAdd(A.count, 1ull);
  if (c >= A.capacity) return;  // cannot happen: capacity = valid pixels of the fused views
  for (int k = 0; k < 3; ++k) {
    A.pos[3 * c + k] = (float)(sx[k] / sw);
    A.nrm[3 * c + k] = (float)(sn[k] / l);
    A.col[3 * c + k] = (unsigned char)sc_clamp(round(sc[k] / sw), 0.0, 255.0);
  }
  A.key[c] = ((unsigned long long)cv.image_id << 32) | ((unsigned long long)(row & 0xffff) << 16) |
             (unsigned long long)(col & 0xffff);
  A.nvis[c] = (unsigned char)write_vis(A.vis + c * A.vis_stride, A.v, hits, nh);
  const unsigned g = cv.idbase + (unsigned)pix;
  A.gid[c] = g;
  A.prio[c] = ((unsigned long long)(~sc_total_key((float)score)) << 32) | (unsigned long long)(g + 1u);
  unsigned* px = A.pix + c * A.pix_stride;
  px[0] = (unsigned)(cv.off + pix);
  for (int i = 0; i < nh; ++i) px[1 + i] = (unsigned)(A.views[hits[i].o].off + hits[i].q);
  A.npix[c] = (unsigned char)(1 + nh);
  A.state[c] = A.mark_used ? 2 : 1;
}

__global__ void k_score_init(const ScoreArgs A, unsigned n) {
  const unsigned i = blockIdx.x * 256u + threadIdx.x;
  if (i == 0) *A.ncur = n;
  if (i < n) const_cast<unsigned*>(A.active)[i] = i;
}

// Adoption rounds (fusion_score.rs:352-414), one kernel per phase.  Phase 1: every undecided candidate frees its
// pixels that are not locked, and one that touches a locked pixel is rejected (the reference rejects it in the next
// phase; locks change only in phase 3, so both see the same locks).
__global__ void __launch_bounds__(256) k_score_reset(const ScoreArgs A) {
  const unsigned n = *A.ncur;
  if (blockIdx.x == 0 && threadIdx.x == 0) *A.nnext = 0;
  for (unsigned t = blockIdx.x * 256u + threadIdx.x; t < n; t += gridDim.x * 256u) {
    const unsigned c = A.active[t];
    const unsigned* px = A.pix + (size_t)c * A.pix_stride;
    const int np = A.npix[c];
    bool locked = false;
    for (int i = 0; i < np; ++i) {
      unsigned long long* cl = A.claim + px[i];
      if (*cl == PS_SCORE_LOCKED)
        locked = true;
      else
        *cl = PS_SCORE_FREE;
    }
    if (locked) A.state[c] = 0;
  }
}
// Phase 2: the undecided candidates claim their pixels by their priority (atomic minimum).
__global__ void __launch_bounds__(256) k_score_claim(const ScoreArgs A) {
  const unsigned n = *A.ncur;
  for (unsigned t = blockIdx.x * 256u + threadIdx.x; t < n; t += gridDim.x * 256u) {
    const unsigned c = A.active[t];
    if (A.state[c] != 2) continue;
    const unsigned* px = A.pix + (size_t)c * A.pix_stride;
    const unsigned long long pr = A.prio[c];
    const int np = A.npix[c];
    for (int i = 0; i < np; ++i) atomicMin(A.claim + px[i], pr);
  }
}
// Phase 3: a candidate that holds all its pixels is adopted and locks them; the other undecided ones go to the next
// round.  A pixel that holds this candidate's priority is claimed by no adopted candidate but this one, so the locks
// written meanwhile by others never touch it: adoption and locking can share the launch.
__global__ void __launch_bounds__(256) k_score_adopt(const ScoreArgs A) {
  const unsigned n = *A.ncur;
  for (unsigned t = blockIdx.x * 256u + threadIdx.x; t < n; t += gridDim.x * 256u) {
    const unsigned c = A.active[t];
    if (A.state[c] != 2) continue;
    const unsigned* px = A.pix + (size_t)c * A.pix_stride;
    const unsigned long long pr = A.prio[c];
    const int np = A.npix[c];
    bool all = true;
    for (int i = 0; i < np; ++i) all = all && A.claim[px[i]] == pr;
    if (all) {
      A.state[c] = 1;
      for (int i = 0; i < np; ++i) A.claim[px[i]] = PS_SCORE_LOCKED;
      atomicAdd(A.adopted, 1ull);
    } else {
      A.next[atomicAdd(A.nnext, 1u)] = c;
    }
  }
}

// Every 97th valid depth of a view in row-major order (one CTA of 1024 threads walks the view in chunks with a block
// scan of the valid flags), then the median of those samples over fx (quantile 0.5: the two middle order statistics,
// interpolated in binary64) by bisection over order-preserving keys.
__device__ __forceinline__ unsigned gsd_key(float f) { return __float_as_uint(f) | 0x80000000u; }  // f > 0
__global__ void __launch_bounds__(1024) k_gsd(const float4* __restrict__ plane, const GsdView* __restrict__ views,
                                              float* samples, unsigned* scount, double* gsd) {
  __shared__ unsigned wsum[32];
  __shared__ unsigned long long red[32];
  const GsdView V = views[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  unsigned g = 0;  // valid pixels before the chunk (uniform)
  for (int c0 = 0; c0 < V.npix; c0 += 1024) {
    const int i = c0 + tid;
    float d = 0.f;
    const bool valid = i < V.npix && (d = plane[V.off + i].w) > 0.0f;
    const unsigned b = __ballot_sync(0xffffffffu, valid);
    if (lane == 0) wsum[warp] = __popc(b);
    __syncthreads();
    unsigned before = 0, total = 0;
    for (int w = 0; w < 32; ++w) {
      if (w < warp) before += wsum[w];
      total += wsum[w];
    }
    const unsigned e = g + before + __popc(b & ((1u << lane) - 1u));
    if (valid && e % 97u == 0u) samples[V.soff + e / 97u] = d;
    g += total;
    __syncthreads();
  }
  const unsigned m = (g + 96u) / 97u;
  if (tid == 0) scount[blockIdx.x] = m;
  if (m == 0) {
    if (tid == 0) gsd[blockIdx.x] = __longlong_as_double(0x7ff8000000000000ll);  // NaN: no valid depth
    return;
  }
  __syncthreads();
  const float* seg = samples + V.soff;
  const double pos = 0.5 * (double)(m - 1u);
  const unsigned lo = (unsigned)floor(pos), hi = min(lo + 1u, m - 1u);
  double val[2];
  for (int s2 = 0; s2 < 2; ++s2) {
    const unsigned k = s2 == 0 ? lo : hi;
    unsigned a = 0u, bnd = 0xffffffffu;
    while (a < bnd) {
      const unsigned mid = a + (bnd - a) / 2u;
      unsigned long long c = 0;
      for (unsigned j = tid; j < m; j += 1024u) c += gsd_key(seg[j]) <= mid;
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      __syncthreads();
      if (lane == 0) red[warp] = c;
      __syncthreads();
      unsigned long long tot = 0;
      for (int w = 0; w < 32; ++w) tot += red[w];
      if (tot >= (unsigned long long)k + 1ull) bnd = mid;
      else a = mid + 1u;
    }
    val[s2] = (double)__uint_as_float(a & 0x7fffffffu);
  }
  if (tid == 0) gsd[blockIdx.x] = (val[0] + (val[1] - val[0]) * (pos - (double)lo)) / V.fx;
}

// One thread per fused point: the candidate views are the overlap lists of its contributing views in order,
// de-duplicated and cut at `limit` (views that were not fused take their place in the count, as in the reference);
// each fused candidate that sees the point in front of its camera at a pixel with a valid depth votes: a violation
// when the point lies in front of that depth by more than tau, a support when it agrees within tau.  The point is
// removed when it has at least min_violations violations and more violations than supports.
__global__ void __launch_bounds__(256) k_visibility(const VisArgs A) {
  const unsigned long long i = (unsigned long long)blockIdx.x * 256ull + threadIdx.x;
  if (i >= A.n) return;
  if (A.masked && A.keep[i] == 0) return;
  const double x[3] = {(double)A.pos[3 * i], (double)A.pos[3 * i + 1], (double)A.pos[3 * i + 2]};
  int cand[PS_VIS_MAX_CHECK];
  int nc = 0;
  bool full = false;
  const unsigned short* vl = A.vis + i * A.vis_stride;
  for (int a = 0; a < (int)A.nvis[i] && !full; ++a) {
    const int v = vl[a];
    if (v >= A.nviews) continue;
    for (int j = A.ovoff[v]; j < A.ovoff[v + 1]; ++j) {
      if (nc >= A.limit) {
        full = true;
        break;
      }
      const int o = A.ovlist[j];
      bool dup = false;
      for (int k = 0; k < nc; ++k) dup = dup || cand[k] == o;
      if (!dup) cand[nc++] = o;
    }
  }
  int viol = 0, sup = 0;
  for (int k = 0; k < nc; ++k) {
    const int v = cand[k];
    if (v < 0 || v >= A.nviews || !A.used[v]) continue;
    const FuseView& c = A.views[v];
    const double* r = c.r;
    const double cx = r[0] * x[0] + r[1] * x[1] + r[2] * x[2] + c.t[0];
    const double cy = r[3] * x[0] + r[4] * x[1] + r[5] * x[2] + c.t[1];
    const double cz = r[6] * x[0] + r[7] * x[1] + r[8] * x[2] + c.t[2];
    if (cz <= 0.0) continue;
    const double col = round(c.k[0] * cx / cz + c.k[2]), row = round(c.k[1] * cy / cz + c.k[3]);
    if (col < 0.0 || row < 0.0 || col >= (double)c.w || row >= (double)c.h) continue;
    const double dv = (double)A.plane[c.off + (long long)row * c.w + (long long)col].w;
    if (dv <= 0.0) continue;
    if (cz < dv * (1.0 - A.tau)) viol++;
    else if (fabs(cz - dv) <= A.tau * dv) sup++;
  }
  const bool keep = !(viol >= A.min_violations && viol > sup);
  A.keep[i] = keep ? 1 : 0;
  if (!keep) atomicAdd(&A.removed[i < A.n1 ? 0 : 1], 1ull);
}

cudaError_t launch_visibility(const VisArgs& A, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  k_visibility<<<(unsigned)((A.n + 255) / 256), 256, 0, st>>>(A);
  return cudaGetLastError();
}

// ---- smoothing along normals ------------------------------------------------------------------------------------
// Cells of size r, packed 21 bits per axis (offset by 2^20) plus one so that 0 marks an empty slot.
#define PS_SM_LIM ((1ll << 20) - 2)
__device__ __forceinline__ unsigned long long sm_code(long long cx, long long cy, long long cz) {
  return ((unsigned long long)(cx + (1ll << 20)) << 42 | (unsigned long long)(cy + (1ll << 20)) << 21 |
          (unsigned long long)(cz + (1ll << 20))) + 1ull;
}
__device__ __forceinline__ bool sm_cell(const SmoothArgs& A, unsigned long long i, long long* c) {
  for (int a = 0; a < 3; ++a) {
    const double f = floor((double)A.pos[3 * i + a] / A.r);
    if (!(f >= (double)-PS_SM_LIM && f <= (double)PS_SM_LIM)) return false;
    c[a] = (long long)f;
  }
  return true;
}
__device__ __forceinline__ unsigned long long sm_order(const SmoothArgs& A, unsigned u) {
  if (A.gid) return (unsigned long long)A.gid[u];
  return ((unsigned long long)(u >= A.n1) << 63) | A.key[u];
}
__device__ __forceinline__ int sm_find(const SmoothArgs& A, unsigned long long code) {
  unsigned slot = (unsigned)(grid_mix(code) & (A.cap - 1u));
  for (unsigned t = 0; t < A.cap; ++t) {
    const unsigned long long k = A.hkeys[slot];
    if (k == code) return (int)slot;
    if (k == 0ull) return -1;
    slot = (slot + 1u) & (A.cap - 1u);
  }
  return -1;
}

__global__ void __launch_bounds__(256) k_sm_insert(const SmoothArgs A) {
  const unsigned long long i = (unsigned long long)blockIdx.x * 256ull + threadIdx.x;
  if (i >= A.n || (A.keep && !A.keep[i])) return;
  long long c[3];
  if (!sm_cell(A, i, c)) {
    atomicExch(A.flag, 1);
    return;
  }
  const unsigned long long code = sm_code(c[0], c[1], c[2]);
  unsigned slot = (unsigned)(grid_mix(code) & (A.cap - 1u));
  for (unsigned t = 0; t < A.cap; ++t) {
    const unsigned long long prev = atomicCAS(&A.hkeys[slot], 0ull, code);
    if (prev == 0ull || prev == code) {
      A.pslot[i] = slot;
      atomicAdd(&A.hcnt[slot], 1u);
      return;
    }
    slot = (slot + 1u) & (A.cap - 1u);
  }
  atomicExch(A.flag, 1);  // cannot happen: the table is at most half full
}
__global__ void __launch_bounds__(256) k_sm_alloc(const SmoothArgs A) {
  const unsigned s = blockIdx.x * 256u + threadIdx.x;
  if (s < A.cap && A.hcnt[s]) A.hstart[s] = atomicAdd(A.total, A.hcnt[s]);
}
__global__ void __launch_bounds__(256) k_sm_scatter(const SmoothArgs A) {
  const unsigned long long i = (unsigned long long)blockIdx.x * 256ull + threadIdx.x;
  if (i >= A.n || (A.keep && !A.keep[i])) return;
  long long c[3];
  if (!sm_cell(A, i, c)) return;
  const unsigned s = A.pslot[i];
  A.list[A.hstart[s] + atomicAdd(&A.hcur[s], 1u)] = (unsigned)i;
}
// each cell's points in cloud order (first pass before second, then ascending key; or ascending candidate number):
// insertion sort per cell
__global__ void __launch_bounds__(256) k_sm_sort(const SmoothArgs A) {
  const unsigned s = blockIdx.x * 256u + threadIdx.x;
  if (s >= A.cap || !A.hcnt[s]) return;
  unsigned* l = A.list + A.hstart[s];
  const unsigned m = A.hcnt[s];
  for (unsigned a = 1; a < m; ++a) {
    const unsigned u = l[a];
    const unsigned long long ku = sm_order(A, u);
    unsigned b = a;
    while (b > 0 && sm_order(A, l[b - 1]) > ku) {
      l[b] = l[b - 1];
      --b;
    }
    l[b] = u;
  }
}
__device__ __forceinline__ void sm_normal(const SmoothArgs& A, unsigned long long i, double* n) {
  const double m[3] = {(double)A.nrm[3 * i], (double)A.nrm[3 * i + 1], (double)A.nrm[3 * i + 2]};
  const double l = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  for (int a = 0; a < 3; ++a) n[a] = l > 1e-12 ? m[a] / l : 0.0;
}
// The move of one point: neighbours in the 27 cells around (z, then y, then x offsets; each cell in cloud order)
// within r, other than the point, whose normal is within the angle, weigh exp(-d²/(2(r/2)²) - dn²/(2σ²)); the point
// moves along its normal by Σ w·dn / (1 + Σ w).
__global__ void __launch_bounds__(256) k_sm_step(const SmoothArgs A) {
  const unsigned long long i = (unsigned long long)blockIdx.x * 256ull + threadIdx.x;
  if (i >= A.n || (A.keep && !A.keep[i])) return;
  long long c[3];
  if (!sm_cell(A, i, c)) return;
  const double pi[3] = {(double)A.pos[3 * i], (double)A.pos[3 * i + 1], (double)A.pos[3 * i + 2]};
  double ni[3];
  sm_normal(A, i, ni);
  double t = 0.0;
  if (!(ni[0] == 0.0 && ni[1] == 0.0 && ni[2] == 0.0)) {
    double sw = 1.0, swd = 0.0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int s = sm_find(A, sm_code(c[0] + dx, c[1] + dy, c[2] + dz));
          if (s < 0) continue;
          const unsigned* l = A.list + A.hstart[s];
          for (unsigned q = 0; q < A.hcnt[s]; ++q) {
            const unsigned j = l[q];
            const double dv[3] = {(double)A.pos[3 * j] - pi[0], (double)A.pos[3 * j + 1] - pi[1],
                                  (double)A.pos[3 * j + 2] - pi[2]};
            const double d2 = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
            if (d2 > A.r2 || j == (unsigned)i) continue;
            double nj[3];
            sm_normal(A, j, nj);
            if (ni[0] * nj[0] + ni[1] * nj[1] + ni[2] * nj[2] < A.cos_n) continue;
            const double dn = ni[0] * dv[0] + ni[1] * dv[1] + ni[2] * dv[2];
            const double w = ps_exp64(-d2 * A.inv_2ss - dn * dn * A.inv_2sr);
            sw += w;
            swd += w * dn;
          }
        }
    t = swd / sw;
  }
  for (int a = 0; a < 3; ++a) A.pos2[3 * i + a] = (float)(pi[a] + t * ni[a]);
}

cudaError_t launch_smooth_pass(const SmoothArgs& A, cudaStream_t st) {
  if (A.n == 0) return cudaSuccess;
  const unsigned gp = (unsigned)((A.n + 255) / 256), gs = (A.cap + 255) / 256;
  k_sm_insert<<<gp, 256, 0, st>>>(A);
  k_sm_alloc<<<gs, 256, 0, st>>>(A);
  k_sm_scatter<<<gp, 256, 0, st>>>(A);
  k_sm_sort<<<gs, 256, 0, st>>>(A);
  k_sm_step<<<gp, 256, 0, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_fuse(const FuseArgs& A, int w, int h, cudaStream_t st) {
  const dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
  k_fuse<<<g, b, 0, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_fuse_second(const FuseArgs& A, int w, int h, int stage, cudaStream_t st) {
  const dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
  k_fuse_second<<<g, b, 0, st>>>(A, stage);
  return cudaGetLastError();
}

cudaError_t launch_score_candidates(const ScoreArgs& A, int w, int h, cudaStream_t st) {
  const dim3 b(32, 8), g((w + 31) / 32, (h + 7) / 8);
  k_score<<<g, b, 0, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_score_init(const ScoreArgs& A, unsigned n, cudaStream_t st) {
  k_score_init<<<(n + 255) / 256 + (n == 0), 256, 0, st>>>(A, n);
  return cudaGetLastError();
}

cudaError_t launch_score_round(const ScoreArgs& A, int blocks, cudaStream_t st) {
  k_score_reset<<<blocks, 256, 0, st>>>(A);
  k_score_claim<<<blocks, 256, 0, st>>>(A);
  k_score_adopt<<<blocks, 256, 0, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_gsd(const float4* plane, const GsdView* views, int nviews, float* samples, unsigned* scount,
                       double* gsd, cudaStream_t st) {
  if (nviews <= 0) return cudaSuccess;
  k_gsd<<<nviews, 1024, 0, st>>>(plane, views, samples, scount, gsd);
  return cudaGetLastError();
}

cudaError_t launch_grid_insert(const float* pos, unsigned n, double cell, unsigned long long* keys, unsigned* heads,
                               unsigned* next, unsigned cap, int* overflow, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  k_grid_insert<<<(n + 255) / 256, 256, 0, st>>>(pos, n, cell, keys, heads, next, cap, overflow);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------- image pyramid
// One level of build_pyramid (crates/dense/src/upsample.rs:46-102): separable 3-tap blur with clamped borders
// (tmp = g0·s[x-1] + g1·s[x] + g2·s[x+1], then the same vertically on tmp, each sum left to right), 2×2 average
// 0.25·(((b00 + b01) + b10) + b11), rounded half away from zero and clamped to u8.  One thread per output pixel
// recomputes the 4 × 2 blurred values it needs (no contraction: the same binary32 operations as the reference).
__device__ __forceinline__ float pyr_src(const unsigned char* in, int w, int h, int y, int x) {
  x = min(max(x, 0), w - 1);
  y = min(max(y, 0), h - 1);
  return (float)in[(long long)y * w + x];
}
__device__ __forceinline__ float pyr_tmp(const unsigned char* in, int w, int h, int y, int x, float g0, float g1,
                                         float g2) {
  return (g0 * pyr_src(in, w, h, y, x - 1) + g1 * pyr_src(in, w, h, y, x)) + g2 * pyr_src(in, w, h, y, x + 1);
}
__device__ __forceinline__ float pyr_blur(const unsigned char* in, int w, int h, int y, int x, float g0, float g1,
                                          float g2) {
  const int ym = max(y - 1, 0), yp = min(y + 1, h - 1);
  return (g0 * pyr_tmp(in, w, h, ym, x, g0, g1, g2) + g1 * pyr_tmp(in, w, h, y, x, g0, g1, g2)) +
         g2 * pyr_tmp(in, w, h, yp, x, g0, g1, g2);
}
__global__ void k_pyramid(const unsigned char* in, int w, int h, unsigned char* out, float g0, float g1, float g2) {
  const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y * blockDim.y + threadIdx.y;
  const int nw = w / 2, nh = h / 2;
  if (X >= nw || Y >= nh) return;
  const int y = 2 * Y, x = 2 * X;
  const float b00 = pyr_blur(in, w, h, y, x, g0, g1, g2), b01 = pyr_blur(in, w, h, y, x + 1, g0, g1, g2);
  const float b10 = pyr_blur(in, w, h, y + 1, x, g0, g1, g2), b11 = pyr_blur(in, w, h, y + 1, x + 1, g0, g1, g2);
  const float v = 0.25f * (((b00 + b01) + b10) + b11);
  out[(long long)Y * nw + X] = (unsigned char)fminf(fmaxf(roundf(v), 0.0f), 255.0f);
}

// ---------------------------------------------------------------------------------------------- hole filling
// 8-bit gray value of an image-plane pixel: planes of 8-bit images hold the correctly rounded u/255, and
// round(255·value) gives u back exactly for every u.
__device__ __forceinline__ int fill_gray(const FillArgs& A, int x, int y) {
  return (int)rintf(A.img[(long long)y * A.pitch + x] * 255.0f);
}

// The fill of every pixel from the unfilled state (postproc.rs:155-193): an invalid pixel with a run cost of at most
// max_cost walks the 8 directions in the reference's order, up to maxd steps, stopping at the border or where the gray
// value jumps by more than `step` from the previous pixel; the first valid pixel met ends a direction, and the one
// with the smallest (|gray difference|, distance) over the directions (the earliest on ties) lends its plane through
// plane_transfer (crates/dense/src/math.rs:146-154, binary64).
__global__ void __launch_bounds__(256) k_fill_find(const FillArgs A) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)A.w * A.h) return;
  const int y = (int)(i / A.w), x = (int)(i - (long long)y * A.w);
  float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
  float oc = 0.f;
  if (!(A.plane[i].w > 0.f) && !(A.cost[i] > A.max_cost)) {
    const int ip = fill_gray(A, x, y);
    const int dxs[8] = {1, -1, 0, 0, 1, -1, 1, -1}, dys[8] = {0, 0, 1, -1, 1, -1, -1, 1};
    bool found = false;
    int bd = 0, bs = 0;
    long long bq = 0;
    for (int d = 0; d < 8; ++d) {
      int prev = ip;
      for (int s = 1; s <= A.maxd; ++s) {
        const int qx = x + dxs[d] * s, qy = y + dys[d] * s;
        if (qx < 0 || qy < 0 || qx >= A.w || qy >= A.h) break;
        const int iq = fill_gray(A, qx, qy);
        if (abs(iq - prev) > A.step) break;
        prev = iq;
        const long long q = (long long)qy * A.w + qx;
        if (A.plane[q].w > 0.f) {
          const int diff = abs(iq - ip);
          if (!found || diff < bd || (diff == bd && s < bs)) {
            found = true;
            bd = diff;
            bs = s;
            bq = q;
          }
          break;
        }
      }
    }
    if (found) {
      const float4 pq = A.plane[bq];
      const double qx = (double)(bq % A.w), qy = (double)(bq / A.w);
      const double rq0 = (qx - A.k[2]) / A.k[0], rq1 = (qy - A.k[3]) / A.k[1];
      const double rp0 = ((double)x - A.k[2]) / A.k[0], rp1 = ((double)y - A.k[3]) / A.k[1];
      const double n0 = (double)pq.x, n1 = (double)pq.y, n2 = (double)pq.z;
      const double num = n0 * rq0 + n1 * rq1 + n2 * 1.0;
      const double den = n0 * rp0 + n1 * rp1 + n2 * 1.0;
      if (!(den > -1e-6)) {
        const double dd = (double)pq.w * num / den;
        if (dd > 0.0 && isfinite(dd)) {
          out = make_float4(pq.x, pq.y, pq.z, (float)dd);
          oc = A.cost[bq];
        }
      }
    }
  }
  A.tplane[i] = out;
  A.tcost[i] = oc;
}

__global__ void __launch_bounds__(256) k_fill_apply(const FillArgs A) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool f = false;
  if (i < (long long)A.w * A.h) {
    const float4 t = A.tplane[i];
    if (t.w > 0.f) {
      A.plane[i] = t;
      A.cost[i] = A.tcost[i];
      f = true;
    }
  }
  const unsigned m = __ballot_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(A.filled, (unsigned long long)__popc(m));
}

cudaError_t launch_fill_holes(const FillArgs& A, cudaStream_t st) {
  const long long n = (long long)A.w * A.h;
  if (n <= 0) return cudaSuccess;
  const unsigned g = (unsigned)((n + 255) / 256);
  k_fill_find<<<g, 256, 0, st>>>(A);
  k_fill_apply<<<g, 256, 0, st>>>(A);
  return cudaGetLastError();
}

// Reference planes of a session: out[y·pitch + x] = lut[in[y·w + x]] (lut = the correctly rounded u/255 of the host,
// so the plane has the bits the oracle's plane has).
__global__ void k_u8_plane(const unsigned char* __restrict__ in, int w, int h, const float* __restrict__ lut,
                           float* __restrict__ out, int pitch) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)w * h) return;
  const int y = (int)(i / w), x = (int)(i - (long long)y * w);
  out[(long long)y * pitch + x] = lut[in[i]];
}

cudaError_t launch_u8_plane(const unsigned char* in, int w, int h, const float* lut, float* out, int pitch,
                            cudaStream_t st) {
  const long long n = (long long)w * h;
  if (n <= 0) return cudaSuccess;
  k_u8_plane<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, w, h, lut, out, pitch);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------- fused cloud order
// Cell of point i (see CloudOrderArgs), or -1 when the point was not kept or its key names no fused view.
__device__ __forceinline__ long long cloud_cell(const CloudOrderArgs& A, unsigned long long i) {
  if (A.keep && !A.keep[i]) return -1;
  if (A.gid) return A.gid[i] < A.cells ? (long long)A.gid[i] : -1;
  const unsigned long long k = A.key[i];
  const unsigned id = (unsigned)(k >> 32);
  const int row = (int)((k >> 16) & 0xffffu), col = (int)(k & 0xffffu);
  if (A.nids <= 0) return -1;
  int lo = 0, hi = A.nids - 1;
  while (lo < hi) {  // the fused views' image ids are ascending and distinct
    const int mid = (lo + hi) >> 1;
    if (A.ids[mid] < id) lo = mid + 1;
    else hi = mid;
  }
  if (A.ids[lo] != id || col >= A.width[lo]) return -1;
  const unsigned long long cell = A.base[lo] + (unsigned long long)row * A.width[lo] + col;
  if (cell >= A.cells) return -1;  // never for keys the fusion kernels write; the grid's bound all the same
  const unsigned long long pass = i < A.count1 ? 0ull : 1ull;
  return (long long)(pass * A.cells + cell);
}

__global__ void __launch_bounds__(256) k_cloud_mark(CloudOrderArgs A) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const long long c = cloud_cell(A, i);
  if (c >= 0) A.rank[c] = 1u;
}

__global__ void __launch_bounds__(256) k_cloud_scatter(CloudOrderArgs A) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const long long c = cloud_cell(A, i);
  if (c < 0) return;
  const unsigned long long j = A.rank[c];
  if (A.opos)
    for (int k = 0; k < 3; ++k) A.opos[3 * j + k] = A.pos[3 * i + k];
  if (A.onrm)
    for (int k = 0; k < 3; ++k) A.onrm[3 * j + k] = A.nrm[3 * i + k];
  if (A.ocol)
    for (int k = 0; k < 3; ++k) A.ocol[3 * j + k] = A.col[3 * i + k];
  if (A.okey) A.okey[j] = A.key[i];
  if (A.onvis) A.onvis[j] = A.nvis[i];
  if (A.ovis)
    for (int t = 0; t < A.ovis_stride; ++t)
      A.ovis[j * A.ovis_stride + t] = t < A.vis_stride && t < A.nvis[i] ? A.vis[i * A.vis_stride + t] : 0;
}

cudaError_t launch_cloud_mark(const CloudOrderArgs& A, cudaStream_t st) {
  if (!A.n) return cudaSuccess;
  k_cloud_mark<<<(unsigned)((A.n + 255) / 256), 256, 0, st>>>(A);
  return cudaGetLastError();
}
cudaError_t launch_cloud_scatter(const CloudOrderArgs& A, cudaStream_t st) {
  if (!A.n) return cudaSuccess;
  k_cloud_scatter<<<(unsigned)((A.n + 255) / 256), 256, 0, st>>>(A);
  return cudaGetLastError();
}

// Exclusive prefix sum: blocks of 1024 threads scan 4096 entries each (4 consecutive entries per thread, then a
// warp-shuffle scan of the thread sums and of the warp totals), write their totals; the totals are scanned the same
// way (recursively), and every entry adds its block's prefix.  The sums count points, so 32 bits suffice.
constexpr int kScanBlock = 4096;

__global__ void __launch_bounds__(1024) k_scan_block(unsigned* data, unsigned long long n, unsigned* sums) {
  __shared__ unsigned warp_tot[32];
  const unsigned long long b0 = (unsigned long long)blockIdx.x * kScanBlock;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  unsigned v[4], s = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const unsigned long long i = b0 + 4ull * t + k;
    v[k] = i < n ? data[i] : 0u;
    s += v[k];
  }
  unsigned inc = s;  // inclusive scan of the thread sums within the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const unsigned w = warp_tot[lane];
    unsigned wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned u = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += u;
    }
    warp_tot[lane] = wi - w;  // exclusive prefix of the warp totals
    if (lane == 31) sums[blockIdx.x] = wi;
  }
  __syncthreads();
  unsigned run = warp_tot[warp] + inc - s;  // exclusive prefix of this thread's first entry within the block
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const unsigned long long i = b0 + 4ull * t + k;
    if (i < n) data[i] = run;
    run += v[k];
  }
}

__global__ void __launch_bounds__(256) k_scan_add(unsigned* data, unsigned long long n, const unsigned* sums) {
  const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) data[i] += sums[i / kScanBlock];
}

size_t scan_scratch(size_t n) {
  size_t total = 0;
  while (n > 1) {
    n = (n + kScanBlock - 1) / kScanBlock;
    total += n;
  }
  return total + 1;
}

cudaError_t scan_exclusive(unsigned* data, size_t n, unsigned* tmp, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const size_t nb = (n + kScanBlock - 1) / kScanBlock;
  k_scan_block<<<(unsigned)nb, 1024, 0, st>>>(data, n, tmp);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || nb == 1) return e;
  if ((e = scan_exclusive(tmp, nb, tmp + nb, st)) != cudaSuccess) return e;
  k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(data, n, tmp);
  return cudaGetLastError();
}

cudaError_t launch_pyramid(const unsigned char* in, int w, int h, unsigned char* out, const float* g,
                           cudaStream_t st) {
  const dim3 b(32, 8), gr((w / 2 + 31) / 32, (h / 2 + 7) / 8);
  if (w / 2 < 1 || h / 2 < 1) return cudaSuccess;
  k_pyramid<<<gr, b, 0, st>>>(in, w, h, out, g[0], g[1], g[2]);
  return cudaGetLastError();
}

}  // namespace ps_post
