// Neighbour (source) views and per-view depth ranges from sparse point tracks on the GPU: PairStats::new,
// PairStats::select / select_diverse and depth_ranges (crates/dense/src/neighbors.rs:44-186), as
// crates/dense/src/densify.rs:224-241 calls them.
//
// Compiled with the parity flags (no contraction, IEEE division and square root): every double expression is
// evaluated as written, in the order the reference writes it, so counts, selections and depth ranges equal the CPU
// restatement's; angles go through CUDA's acos and atan2 (the reference: the platform's), rounded to binary32 as the
// reference stores them.
//
// Layout: the pairs of n views are a dense n×n table indexed min(a,b)·n + max(a,b) (n <= 4096).  Pass 0 counts the
// pairs of every track, a one-CTA scan turns the counts into segment offsets (and lists the non-empty pairs in
// ascending order), pass 1 writes each pair's angles into its segment, and one CTA per non-empty pair finds the two
// order statistics around 0.75·(m-1) exactly (radix select over order-preserving keys; no sort).  Depth observations
// follow the same count / scan / scatter / order-statistic scheme per view.  One CTA per view then selects its
// sources: candidates gated by the 75th-percentile angle, repeatedly the best by (score, shared count, lower index).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "patchstereo.h"

namespace {

constexpr int NB_NT = 256;
constexpr double NB_PI = 3.141592653589793;  // the binary64 nearest pi
constexpr uint32_t NB_MAX_VIEWS = 4096;

struct NbView {
  double r[9], t[3], c[3];
};

// DenseView::center (crates/dense/src/scene.rs:82-89): -(Rᵀ t).
__global__ void k_nb_views(const ps_sparse_view* in, int nv, NbView* out) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  NbView o;
  for (int k = 0; k < 9; ++k) o.r[k] = in[v].r[k];
  for (int k = 0; k < 3; ++k) o.t[k] = in[v].t[k];
  for (int j = 0; j < 3; ++j) o.c[j] = -(o.r[0 * 3 + j] * o.t[0] + o.r[1 * 3 + j] * o.t[1] + o.r[2 * 3 + j] * o.t[2]);
  out[v] = o;
}

// Triangulation angle of a point seen from two centres, min(a, pi - a) (neighbors.rs:55-69), stored in binary32.
__device__ float nb_angle(const double* x, const double* ca, const double* cb) {
  const double u[3] = {ca[0] - x[0], ca[1] - x[1], ca[2] - x[2]};
  const double w[3] = {cb[0] - x[0], cb[1] - x[1], cb[2] - x[2]};
  const double nu = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  const double nw = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  double ang = 0.0;
  if (!(nu == 0.0 || nw == 0.0)) {
    double c = (u[0] * w[0] + u[1] * w[1] + u[2] * w[2]) / (nu * nw);
    if (c < -1.0) c = -1.0;
    else if (c > 1.0) c = 1.0;
    const double t = acos(c);
    ang = fmin(t, NB_PI - t);
  }
  return (float)ang;
}

// Pass 0 counts every pair of distinct entries of every track (repeated views of a track count as the reference
// counts them); pass 1 writes the pair's angle into the pair's segment.
__global__ void __launch_bounds__(NB_NT) k_nb_pairs(const NbView* __restrict__ views, int nv,
                                                    const double* __restrict__ xyz, const uint32_t* __restrict__ toff,
                                                    const uint32_t* __restrict__ tview, long long np, int pass,
                                                    unsigned* cnt, const unsigned long long* __restrict__ off,
                                                    unsigned* cursor, float* ang) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += stride) {
    const uint32_t b0 = toff[p], b1 = toff[p + 1];
    const double x[3] = {xyz[3 * p], xyz[3 * p + 1], xyz[3 * p + 2]};
    for (uint32_t i = b0; i < b1; ++i)
      for (uint32_t j = b0; j < i; ++j) {
        const uint32_t a = tview[i], b = tview[j];
        if (a == b) continue;
        const size_t key = (size_t)min(a, b) * nv + max(a, b);
        if (pass == 0) atomicAdd(&cnt[key], 1u);
        else ang[off[key] + atomicAdd(&cursor[key], 1u)] = nb_angle(x, views[a].c, views[b].c);
      }
  }
}

// Depth of every observation in its view (the third camera coordinate, neighbors.rs:160-173); pass 0 counts the
// positive ones per view, pass 1 writes them into the view's segment.
__global__ void __launch_bounds__(NB_NT) k_nb_depths(const NbView* __restrict__ views, const double* __restrict__ xyz,
                                                     const uint32_t* __restrict__ toff,
                                                     const uint32_t* __restrict__ tview, long long np, int pass,
                                                     unsigned* cnt, const unsigned long long* __restrict__ off,
                                                     unsigned* cursor, double* dep) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += stride) {
    const double x[3] = {xyz[3 * p], xyz[3 * p + 1], xyz[3 * p + 2]};
    for (uint32_t i = toff[p]; i < toff[p + 1]; ++i) {
      const uint32_t v = tview[i];
      const NbView& w = views[v];
      const double d = w.r[6] * x[0] + w.r[7] * x[1] + w.r[8] * x[2] + w.t[2];
      if (!(d > 0.0)) continue;
      if (pass == 0) atomicAdd(&cnt[v], 1u);
      else dep[off[v] + atomicAdd(&cursor[v], 1u)] = d;
    }
  }
}

// Exclusive prefix sums of cnt[0..n) into off and the ascending list of indices with cnt > 0 into nz; one CTA of 1024
// threads walks the array in chunks (Hillis-Steele scan per chunk).
__global__ void __launch_bounds__(1024) k_nb_scan(const unsigned* __restrict__ cnt, size_t n, unsigned long long* off,
                                                  unsigned* nz, unsigned* nnz, unsigned long long* total) {
  __shared__ unsigned long long ssum[1024];
  __shared__ unsigned sflag[1024];
  unsigned long long base = 0;
  unsigned nzbase = 0;
  for (size_t c0 = 0; c0 < n; c0 += 1024) {
    const size_t i = c0 + threadIdx.x;
    const unsigned v = i < n ? cnt[i] : 0u;
    ssum[threadIdx.x] = v;
    sflag[threadIdx.x] = v ? 1u : 0u;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
      const unsigned long long a = (int)threadIdx.x >= d ? ssum[threadIdx.x - d] : 0ull;
      const unsigned b = (int)threadIdx.x >= d ? sflag[threadIdx.x - d] : 0u;
      __syncthreads();
      ssum[threadIdx.x] += a;
      sflag[threadIdx.x] += b;
      __syncthreads();
    }
    if (i < n) {
      off[i] = base + ssum[threadIdx.x] - v;
      if (v) nz[nzbase + sflag[threadIdx.x] - 1] = (unsigned)i;
    }
    const unsigned long long csum = ssum[1023];
    const unsigned cnz = sflag[1023];
    __syncthreads();
    base += csum;
    nzbase += cnz;
  }
  if (threadIdx.x == 0) {
    *total = base;
    *nnz = nzbase;
  }
}

// Order-preserving unsigned keys of binary32 / binary64 values (negative values reversed below the positives).
__device__ __forceinline__ unsigned key32(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unkey32(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
__device__ __forceinline__ unsigned long long key64(double f) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(f);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double unkey64(unsigned long long k) {
  return __longlong_as_double((long long)((k >> 63) ? (k & 0x7fffffffffffffffull) : ~k));
}

// The k-th smallest (0-based) of seg[0..m) by radix select over the order-preserving keys: 8-bit digits from the
// most significant; each pass counts, in a shared histogram, the digit of every key that agrees with the digits
// chosen so far, and takes the digit whose running count passes k (4 passes for binary32, 8 for binary64).  Every
// thread of the CTA returns it.
template <typename T, typename K, typename KeyFn>
__device__ K radix_kth(const T* seg, unsigned m, unsigned k, KeyFn key, unsigned* hist, K* chosen) {
  constexpr int NB = (int)sizeof(K) * 8;
  K prefix = 0, mask = 0;
  unsigned rank = k;
  for (int shift = NB - 8; shift >= 0; shift -= 8) {
    for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d] = 0u;
    __syncthreads();
    for (unsigned i = threadIdx.x; i < m; i += blockDim.x) {
      const K kk = key(seg[i]);
      if ((kk & mask) == prefix) atomicAdd(&hist[(unsigned)(kk >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned cum = 0, d = 0;
      for (; d < 255u && cum + hist[d] <= rank; ++d) cum += hist[d];
      chosen[0] = (K)d;
      chosen[1] = (K)(rank - cum);
    }
    __syncthreads();
    prefix |= chosen[0] << shift;
    mask |= (K)255 << shift;
    rank = (unsigned)chosen[1];
    __syncthreads();
  }
  return prefix;
}
__device__ float kth32(const float* seg, unsigned m, unsigned k, unsigned* hist, unsigned* chosen) {
  return unkey32(radix_kth<float, unsigned>(seg, m, k, [](float f) { return key32(f); }, hist, chosen));
}
__device__ double kth64(const double* seg, unsigned m, unsigned k, unsigned* hist, unsigned long long* chosen) {
  return unkey64(radix_kth<double, unsigned long long>(seg, m, k, [](double f) { return key64(f); }, hist, chosen));
}

// quantile_sorted(angles, 0.75) of every non-empty pair (crates/dense/src/math.rs:126-135): the order statistics at
// floor(0.75·(m-1)) and the next, interpolated in binary64.
__global__ void __launch_bounds__(NB_NT) k_nb_q75(const unsigned* __restrict__ nz, const unsigned* __restrict__ cnt,
                                                  const unsigned long long* __restrict__ off,
                                                  const float* __restrict__ ang, double* q75) {
  __shared__ unsigned hist[256];
  __shared__ unsigned chosen[2];
  const unsigned key = nz[blockIdx.x];
  const unsigned m = cnt[key];
  const float* seg = ang + off[key];
  const double pos = 0.75 * (double)(m - 1u);
  const unsigned lo = (unsigned)floor(pos);
  const unsigned hi = min(lo + 1u, m - 1u);
  const double f = pos - (double)lo;
  const double vlo = (double)kth32(seg, m, lo, hist, chosen);
  const double vhi = hi == lo ? vlo : (double)kth32(seg, m, hi, hist, chosen);
  if (threadIdx.x == 0) q75[key] = vlo + (vhi - vlo) * f;
}

// depth_range_of (neighbors.rs:176-186): the order statistics at floor(0.01·n) and floor(0.99·n) (clamped to n-1),
// times 0.75 and 1.25.
__global__ void __launch_bounds__(NB_NT) k_nb_range(const unsigned* __restrict__ cnt,
                                                    const unsigned long long* __restrict__ off,
                                                    const double* __restrict__ dep, double* range, uint8_t* has) {
  __shared__ unsigned hist[256];
  __shared__ unsigned long long chosen[2];
  const int v = blockIdx.x;
  const unsigned n = cnt[v];
  if (n == 0) {
    if (threadIdx.x == 0) {
      has[v] = 0;
      range[2 * v] = range[2 * v + 1] = 0.0;
    }
    return;
  }
  const double* seg = dep + off[v];
  const unsigned ilo = min((unsigned)floor((double)n * 0.01), n - 1u);
  const unsigned ihi = min((unsigned)floor((double)n * 0.99), n - 1u);
  const double lo = kth64(seg, n, ilo, hist, chosen);
  const double hi = kth64(seg, n, ihi, hist, chosen);
  if (threadIdx.x == 0) {
    has[v] = 1;
    range[2 * v] = 0.75 * lo;
    range[2 * v + 1] = 1.25 * hi;
  }
}

// f64::powi as lowered for a run-time exponent: square-and-multiply over the exponent's bits, lowest bit first.
__device__ double nb_powi(double a, int b) {
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

// One CTA per reference view r: PairStats::select (neighbors.rs:82-101) — candidates o != r with shared points and,
// when min_angle > 0, a 75th-percentile angle of at least min_angle, in descending shared count, ascending index —
// or, with decay < 1, select_diverse (neighbors.rs:108-150): the greedy choice of the highest count·decay^k, k the
// number already taken from the candidate's baseline-azimuth sector (first in the count order on ties).
__global__ void __launch_bounds__(NB_NT) k_nb_select(const NbView* __restrict__ views, int nv,
                                                     const unsigned* __restrict__ cnt, const double* __restrict__ q75,
                                                     double min_angle, unsigned maxn, int diverse, int bins,
                                                     double decay, unsigned* sources, unsigned* nsrc) {
  extern __shared__ unsigned char nb_sh[];
  unsigned* ccnt = reinterpret_cast<unsigned*>(nb_sh);                      // candidate counts (0: not / taken)
  unsigned short* cbin = reinterpret_cast<unsigned short*>(ccnt + nv);     // sector of each candidate
  __shared__ int used[NB_NT + 1];
  __shared__ double ws[NB_NT / 32];
  __shared__ unsigned wc[NB_NT / 32], wo[NB_NT / 32];
  __shared__ unsigned pick_o;
  const int r = blockIdx.x;
  const NbView& vr = views[r];
  for (int o = threadIdx.x; o < nv; o += blockDim.x) {
    unsigned c = 0;
    unsigned short b = 0;
    if (o != r) {
      const size_t key = (size_t)min(r, o) * nv + max(r, o);
      c = cnt[key];
      if (c && min_angle > 0.0 && q75[key] < min_angle) c = 0;
      if (c && diverse) {
        const double* co = views[o].c;
        const double d[3] = {co[0] - vr.c[0], co[1] - vr.c[1], co[2] - vr.c[2]};
        double bb[3];
        for (int k = 0; k < 3; ++k) bb[k] = vr.r[k * 3 + 0] * d[0] + vr.r[k * 3 + 1] * d[1] + vr.r[k * 3 + 2] * d[2];
        const double lat = sqrt(bb[0] * bb[0] + bb[1] * bb[1]);
        if (lat < 0.3 * fabs(bb[2])) {
          b = (unsigned short)bins;
        } else {
          const double a = atan2(bb[1], bb[0]) + NB_PI;
          b = (unsigned short)min((unsigned long long)(a / (2.0 * NB_PI) * (double)bins), (unsigned long long)(bins - 1));
        }
      }
    }
    ccnt[o] = c;
    cbin[o] = b;
  }
  for (int k = threadIdx.x; k <= bins; k += blockDim.x) used[k] = 0;
  __syncthreads();
  unsigned n_out = 0;
  for (unsigned pick = 0; pick < maxn; ++pick) {
    // best of this thread's candidates by (score desc, count desc, index asc); none: count 0
    double bs = 0.0;
    unsigned bc = 0, bo = 0xffffffffu;
    for (int o = threadIdx.x; o < nv; o += blockDim.x) {
      const unsigned c = ccnt[o];
      if (!c) continue;
      const double s = diverse ? (double)c * nb_powi(decay, used[cbin[o]]) : (double)c;
      if (!bc || s > bs || (s == bs && (c > bc || (c == bc && (unsigned)o < bo)))) {
        bs = s;
        bc = c;
        bo = (unsigned)o;
      }
    }
    for (int sh = 16; sh > 0; sh >>= 1) {
      const double s2 = __shfl_xor_sync(0xffffffffu, bs, sh);
      const unsigned c2 = __shfl_xor_sync(0xffffffffu, bc, sh), o2 = __shfl_xor_sync(0xffffffffu, bo, sh);
      if (c2 && (!bc || s2 > bs || (s2 == bs && (c2 > bc || (c2 == bc && o2 < bo))))) {
        bs = s2;
        bc = c2;
        bo = o2;
      }
    }
    if ((threadIdx.x & 31) == 0) {
      ws[threadIdx.x >> 5] = bs;
      wc[threadIdx.x >> 5] = bc;
      wo[threadIdx.x >> 5] = bo;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double s = 0.0;
      unsigned c = 0, o = 0xffffffffu;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
        if (wc[w] && (!c || ws[w] > s || (ws[w] == s && (wc[w] > c || (wc[w] == c && wo[w] < o))))) {
          s = ws[w];
          c = wc[w];
          o = wo[w];
        }
      pick_o = c ? o : 0xffffffffu;
      if (c) {
        sources[(size_t)r * maxn + pick] = o;
        used[cbin[o]]++;
        ccnt[o] = 0;
      }
    }
    __syncthreads();
    if (pick_o == 0xffffffffu) break;
    n_out++;
  }
  for (unsigned k = n_out + threadIdx.x; k < maxn; k += blockDim.x) sources[(size_t)r * maxn + k] = 0xffffffffu;
  if (threadIdx.x == 0) nsrc[r] = n_out;
}

}  // namespace

extern "C" {

void ps_neighbor_params_default(ps_neighbor_params* out) {
  if (!out) return;
  out->num_views = 10;
  out->direction_bins = 8;
  out->min_triangulation_angle_deg = 1.0;
  out->diversity_decay = 1.0;
}

int ps_select_neighbors(int device, const ps_sparse_view* views, uint32_t num_views, const double* xyz,
                        const uint32_t* track_offsets, const uint32_t* track_views, uint64_t num_points,
                        const ps_neighbor_params* p, uint32_t* sources, uint32_t* num_sources, double* depth_range,
                        uint8_t* has_range, uint32_t* pair_count, double* pair_angle75) {
  if (!views || !p || !sources || !num_sources || !depth_range || !has_range) return PS_EINVAL;
  if (num_views < 1 || num_views > NB_MAX_VIEWS || p->num_views < 1 || p->num_views > 1024) return PS_EINVAL;
  if (p->direction_bins > NB_NT) return PS_EINVAL;
  if (num_points && (!xyz || !track_offsets || !track_views)) return PS_EINVAL;
  if (num_points > 0x7fffffffull) return PS_EINVAL;
  // the tracks are read on the device: every offset and view index is checked here first
  const uint64_t nobs = num_points ? track_offsets[num_points] : 0;
  if (num_points && track_offsets[0] != 0) return PS_EINVAL;
  for (uint64_t i = 0; i < num_points; ++i)
    if (track_offsets[i + 1] < track_offsets[i]) return PS_EINVAL;
  for (uint64_t k = 0; k < nobs; ++k)
    if (track_views[k] >= num_views) return PS_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return PS_ENODEV;
  const int nv = (int)num_views;
  const size_t nn = (size_t)nv * nv;
  const int bins = (int)std::max<uint32_t>(p->direction_bins, 1);
  std::vector<void*> bufs;
  auto dev = [&](size_t bytes) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(bytes, 16)) != cudaSuccess) return (void*)nullptr;
    bufs.push_back(q);
    return q;
  };
  cudaStream_t st = nullptr;
  int rc = PS_OK;
  do {
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
      rc = PS_ECUDA;
      break;
    }
    ps_sparse_view* d_in = (ps_sparse_view*)dev(sizeof(ps_sparse_view) * nv);
    NbView* d_v = (NbView*)dev(sizeof(NbView) * nv);
    double* d_xyz = (double*)dev(sizeof(double) * 3 * num_points);
    uint32_t* d_off = (uint32_t*)dev(sizeof(uint32_t) * (num_points + 1));
    uint32_t* d_tv = (uint32_t*)dev(sizeof(uint32_t) * nobs);
    unsigned* d_cnt = (unsigned*)dev(sizeof(unsigned) * nn);
    unsigned* d_cur = (unsigned*)dev(sizeof(unsigned) * nn);
    unsigned long long* d_poff = (unsigned long long*)dev(sizeof(unsigned long long) * nn);
    unsigned* d_nz = (unsigned*)dev(sizeof(unsigned) * nn);
    double* d_q75 = (double*)dev(sizeof(double) * nn);
    unsigned* d_dcnt = (unsigned*)dev(sizeof(unsigned) * nv);
    unsigned* d_dcur = (unsigned*)dev(sizeof(unsigned) * nv);
    unsigned long long* d_doff = (unsigned long long*)dev(sizeof(unsigned long long) * nv);
    unsigned* d_dnz = (unsigned*)dev(sizeof(unsigned) * nv);
    unsigned* d_scal = (unsigned*)dev(64);  // nnz (pairs), nnz (views), totals (8-byte aligned at 16, 24)
    double* d_range = (double*)dev(sizeof(double) * 2 * nv);
    uint8_t* d_has = (uint8_t*)dev((size_t)nv);
    unsigned* d_src = (unsigned*)dev(sizeof(unsigned) * (size_t)nv * p->num_views);
    unsigned* d_nsrc = (unsigned*)dev(sizeof(unsigned) * nv);
    if (bufs.size() != 19) {
      rc = PS_ENOMEM;
      break;
    }
    unsigned long long* d_tot = (unsigned long long*)((char*)d_scal + 16);
    unsigned long long* d_dtot = (unsigned long long*)((char*)d_scal + 24);
    bool ok = cudaMemcpyAsync(d_in, views, sizeof(ps_sparse_view) * nv, cudaMemcpyHostToDevice, st) == cudaSuccess;
    if (num_points) {
      ok = ok && cudaMemcpyAsync(d_xyz, xyz, sizeof(double) * 3 * num_points, cudaMemcpyHostToDevice, st) == cudaSuccess;
      ok = ok && cudaMemcpyAsync(d_off, track_offsets, sizeof(uint32_t) * (num_points + 1), cudaMemcpyHostToDevice, st) ==
                     cudaSuccess;
      ok = ok && cudaMemcpyAsync(d_tv, track_views, sizeof(uint32_t) * nobs, cudaMemcpyHostToDevice, st) == cudaSuccess;
    }
    ok = ok && cudaMemsetAsync(d_cnt, 0, sizeof(unsigned) * nn, st) == cudaSuccess;
    ok = ok && cudaMemsetAsync(d_cur, 0, sizeof(unsigned) * nn, st) == cudaSuccess;
    ok = ok && cudaMemsetAsync(d_q75, 0, sizeof(double) * nn, st) == cudaSuccess;
    ok = ok && cudaMemsetAsync(d_dcnt, 0, sizeof(unsigned) * nv, st) == cudaSuccess;
    ok = ok && cudaMemsetAsync(d_dcur, 0, sizeof(unsigned) * nv, st) == cudaSuccess;
    if (!ok) {
      rc = PS_ECUDA;
      break;
    }
    k_nb_views<<<(nv + 127) / 128, 128, 0, st>>>(d_in, nv, d_v);
    const long long np = (long long)num_points;
    const int grid = (int)std::min<long long>(std::max<long long>((np + NB_NT - 1) / NB_NT, 1), 148 * 16);
    if (np) {
      k_nb_pairs<<<grid, NB_NT, 0, st>>>(d_v, nv, d_xyz, d_off, d_tv, np, 0, d_cnt, nullptr, nullptr, nullptr);
      k_nb_depths<<<grid, NB_NT, 0, st>>>(d_v, d_xyz, d_off, d_tv, np, 0, d_dcnt, nullptr, nullptr, nullptr);
    }
    k_nb_scan<<<1, 1024, 0, st>>>(d_cnt, nn, d_poff, d_nz, d_scal, d_tot);
    k_nb_scan<<<1, 1024, 0, st>>>(d_dcnt, (size_t)nv, d_doff, d_dnz, d_scal + 1, d_dtot);
    unsigned long long tot[2] = {0, 0};
    unsigned nnz = 0;
    ok = cudaGetLastError() == cudaSuccess;
    ok = ok && cudaMemcpyAsync(tot, d_tot, 16, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(&nnz, d_scal, 4, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) {
      rc = PS_ECUDA;
      break;
    }
    float* d_ang = (float*)dev(sizeof(float) * tot[0]);
    double* d_dep = (double*)dev(sizeof(double) * tot[1]);
    if (bufs.size() != 21) {
      rc = PS_ENOMEM;
      break;
    }
    if (np) {
      k_nb_pairs<<<grid, NB_NT, 0, st>>>(d_v, nv, d_xyz, d_off, d_tv, np, 1, d_cnt, d_poff, d_cur, d_ang);
      k_nb_depths<<<grid, NB_NT, 0, st>>>(d_v, d_xyz, d_off, d_tv, np, 1, d_dcnt, d_doff, d_dcur, d_dep);
    }
    if (nnz) k_nb_q75<<<nnz, NB_NT, 0, st>>>(d_nz, d_cnt, d_poff, d_ang, d_q75);
    k_nb_range<<<nv, NB_NT, 0, st>>>(d_dcnt, d_doff, d_dep, d_range, d_has);
    const double min_angle = p->min_triangulation_angle_deg * (NB_PI / 180.0);  // f64::to_radians
    const size_t smem = (size_t)nv * (sizeof(unsigned) + sizeof(unsigned short));
    k_nb_select<<<nv, NB_NT, smem, st>>>(d_v, nv, d_cnt, d_q75, min_angle, p->num_views,
                                         p->diversity_decay < 1.0 ? 1 : 0, bins, p->diversity_decay, d_src, d_nsrc);
    ok = cudaGetLastError() == cudaSuccess;
    ok = ok && cudaMemcpyAsync(sources, d_src, sizeof(unsigned) * (size_t)nv * p->num_views, cudaMemcpyDeviceToHost,
                               st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(num_sources, d_nsrc, sizeof(unsigned) * nv, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(depth_range, d_range, sizeof(double) * 2 * nv, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(has_range, d_has, (size_t)nv, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    if (pair_count)
      ok = ok && cudaMemcpyAsync(pair_count, d_cnt, sizeof(unsigned) * nn, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    if (pair_angle75)
      ok = ok && cudaMemcpyAsync(pair_angle75, d_q75, sizeof(double) * nn, cudaMemcpyDeviceToHost, st) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(st) == cudaSuccess;
    if (!ok) rc = PS_ECUDA;
  } while (false);
  for (void* q : bufs) cudaFree(q);
  if (st) cudaStreamDestroy(st);
  cudaGetLastError();
  return rc;
}

}  // extern "C"
