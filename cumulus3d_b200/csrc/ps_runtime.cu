// Host runtime of the B200 PatchStereo engine and its C ABI (include/patchstereo.h).
//
// It plays the role of the reference's CUDA session (crates/cuda/src/patchmatch.rs:285-1009): one session per
// backend, one stream per session, every image of every level resident in HBM for the session's lifetime.  The
// B200 design differs in these points:
//   * images are uploaded once as normalised f32 planes with a zero border (no CUDA arrays / texture objects);
//   * per-pixel state lives in per-level "slots" (plane float4, cost, best view, count, prior) that persist across
//     calls, so the host-state calls (ps_run, ps_evaluate, …) are thin wrappers over resident ones and a caller that
//     keeps everything on the device (ps_run_resident, ps_snapshot_capture, ps_filter_resident) never copies states;
//   * the FP64 homography setup A = K_j R K^-1, b = K_j t runs on the device once per session;
//   * the batch table rides in the kernel parameters, tiles of all views of a batch are flattened into one grid.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <omp.h>
#include <algorithm>
#include <limits>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/patchstereo.h"
#include "ps_cnn.h"
#include "ps_consts.h"
#include "ps_post.h"
#include "ps_types.h"

#define PS_DECLARE_LAUNCHERS(NS)                                                                           \
  namespace NS {                                                                                           \
  cudaError_t launch_half(const PsRun& P, unsigned tuning, cudaStream_t st);                               \
  bool half_run_ok(unsigned tuning, int wr, int ws);                                                       \
  cudaError_t launch_half_run(const PsRun& P, unsigned tuning, cudaStream_t st);                           \
  int half_lanes(unsigned tuning);                                                                         \
  cudaError_t launch_eval(const PsRun& P, bool tex, cudaStream_t st);                                      \
  cudaError_t launch_filter(const PsRun& P, bool tex, cudaStream_t st);                                    \
  cudaError_t launch_upsample(const PsRun& P, cudaStream_t st);                                            \
  cudaError_t launch_median(const PsRun& P, cudaStream_t st);                                              \
  cudaError_t launch_snapshot(const PsRun& P, float* snap, cudaStream_t st);                               \
  cudaError_t launch_readout(const PsRun& P, float4* out, cudaStream_t st);                                \
  cudaError_t launch_sweep(const PsRun& P, bool tex, cudaStream_t st);                                     \
  cudaError_t launch_restore(const PsRun& P, const float4* up, const float* cinit, float thr, cudaStream_t st); \
  cudaError_t launch_fp32_probe(float* out, int blocks, int iters, cudaStream_t st);                       \
  cudaError_t launch_rcp_check(int e_lo, int e_hi, unsigned long long* bad, unsigned* first, cudaStream_t st); \
  cudaError_t prepare();                                                                                   \
  cudaError_t launch_setup_lpairs(const PsLevel* lv, const PsPair* pairs, const double* pairs64,           \
                                  const int* has64, PsLPair* out, int nviews, int nlevels, cudaStream_t st); \
  }
PS_DECLARE_LAUNCHERS(ps_parity)
PS_DECLARE_LAUNCHERS(ps_fast)
PS_DECLARE_LAUNCHERS(ps_checked)

namespace {

struct Launchers {
  cudaError_t (*half)(const PsRun&, unsigned, cudaStream_t);
  cudaError_t (*eval)(const PsRun&, bool, cudaStream_t);
  cudaError_t (*filter)(const PsRun&, bool, cudaStream_t);
  cudaError_t (*upsample)(const PsRun&, cudaStream_t);
  cudaError_t (*median)(const PsRun&, cudaStream_t);
  cudaError_t (*snapshot)(const PsRun&, float*, cudaStream_t);
  cudaError_t (*readout)(const PsRun&, float4*, cudaStream_t);
  int (*half_lanes)(unsigned);
  cudaError_t (*sweep)(const PsRun&, bool, cudaStream_t);
  cudaError_t (*restore)(const PsRun&, const float4*, const float*, float, cudaStream_t);
  bool (*half_run_ok)(unsigned, int, int);
  cudaError_t (*half_run)(const PsRun&, unsigned, cudaStream_t);
};
const Launchers kParity = {ps_parity::launch_half,     ps_parity::launch_eval,   ps_parity::launch_filter,
                           ps_parity::launch_upsample, ps_parity::launch_median, ps_parity::launch_snapshot,
                           ps_parity::launch_readout,  ps_parity::half_lanes,    ps_parity::launch_sweep,
                           ps_parity::launch_restore, ps_parity::half_run_ok, ps_parity::launch_half_run};
const Launchers kFast = {ps_fast::launch_half,     ps_fast::launch_eval,   ps_fast::launch_filter,
                         ps_fast::launch_upsample, ps_fast::launch_median, ps_fast::launch_snapshot,
                         ps_fast::launch_readout,  ps_fast::half_lanes,    ps_fast::launch_sweep,
                         ps_fast::launch_restore, ps_fast::half_run_ok, ps_fast::launch_half_run};
const Launchers kChecked = {ps_checked::launch_half,     ps_checked::launch_eval,   ps_checked::launch_filter,
                            ps_checked::launch_upsample, ps_checked::launch_median, ps_checked::launch_snapshot,
                            ps_checked::launch_readout,  ps_checked::half_lanes,    ps_checked::launch_sweep,
                            ps_checked::launch_restore, ps_checked::half_run_ok, ps_checked::launch_half_run};

struct PsError {
  int code;
  std::string msg;
};

inline size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Per-level resident state of every view.
struct Slot {
  bool ready = false;
  std::vector<long long> off;  // per view pixel offset
  long long total = 0;
  float4* plane = nullptr;
  float4* aux = nullptr;    // second plane buffer (median input, readout output)
  float4* prior = nullptr;  // coarse-scale candidates
  float* cost = nullptr;
  unsigned char* bview = nullptr;
  unsigned char* count = nullptr;
  std::vector<char> prior_valid;
  float4* proposal = nullptr;  // learned proposals (allocated by the first proposal call of the level)
  float* pconf = nullptr;      // their confidences
  std::vector<char> proposal_valid;
  int* spk = nullptr;          // speckle removal: parent, size, lo, hi, cnt per pixel (5 ints each, lazily)
  unsigned char* marks = nullptr;  // fusion "used" marks
  unsigned char* consumed = nullptr;  // fusion second pass: pixels used by first-pass points
  float* cinit = nullptr;          // multi-scale driver: cost of the upsampled planes
};

// Fused point cloud of the last ps_fuse_resident call (device).
struct FusedCloud {
  unsigned long long cap = 0, count = 0, count1 = 0;  // count1: points of the first pass (they come first)
  // visibility filter: per emitted point 1 = kept (NULL: no filter ran), and the removed points of each pass
  unsigned char* keep = nullptr;
  unsigned long long removed1 = 0, removed2 = 0;
  // score fusion: candidates that lost to a higher-priority one (keep = 0), and each point's candidate number, whose
  // order is the output order (NULL: key order per pass)
  unsigned long long rejected = 0;
  unsigned* gid = nullptr;
  int vis_stride = 0;
  float* pos = nullptr;
  float* nrm = nullptr;
  unsigned char* col = nullptr;
  unsigned long long* key = nullptr;
  unsigned char* nvis = nullptr;
  unsigned short* vis = nullptr;
  unsigned long long* counter = nullptr;
  ps_post::FuseView* views = nullptr;
  // output order on the device (ps_fused_points): cells per pass and, for consistency fusion, the fused views in
  // ascending image id with their first cell and width; `ordered` is false when two fused views share an image id
  unsigned long long cells = 0;
  std::vector<unsigned> ids;
  std::vector<unsigned long long> bases;
  std::vector<int> widths;
  bool ordered = false;
  template <typename Free>
  void release(Free&& free) {
    free(keep);
    free(gid);
    free(pos);
    free(nrm);
    free(col);
    free(key);
    free(nvis);
    free(vis);
    *this = FusedCloud{counter, views};
  }
  FusedCloud() = default;
  FusedCloud(unsigned long long* c, ps_post::FuseView* v) : counter(c), views(v) {}
};

}  // namespace

struct ps_backend {
  int device = 0;
  ps_options opts{};
  std::string name;
  std::string err;
  std::mutex mu;
  bool busy = false;
  // Memory kept between sessions (one session at a time): device buffers come from this stream-ordered pool, which
  // keeps what a session frees for the next one, and the pinned staging buffer passes from session to session.
  cudaMemPool_t pool = nullptr;
  void* pin = nullptr;
  size_t pin_cap = 0;
  // texture arrays of the previous session, reused by size and format (freeing an array can stall for a long time)
  struct CachedArray {
    cudaArray_t a;
    int w, h;
    bool u8;
  };
  std::vector<CachedArray> arrays;
  // host-side failure injection (ps_backend_inject_failure): kind and the successes left before the failure
  uint32_t inject_kind = PS_INJECT_NONE;
  uint32_t inject_after = 0;
};

struct ps_session {
  ps_backend* be = nullptr;
  std::string err;
  cudaStream_t st = nullptr;
  const Launchers* L = &kParity;
  unsigned long long* fault = nullptr;  // checked build: the kernels' fault word (device), else null
  unsigned* qbuf = nullptr;             // persistent half step: queue counter, error word, per-phase done counts
  std::vector<cudaEvent_t> xfer;        // per-view copy events of the host-state transfers (pack/unpack overlap)
  cudaStream_t up = nullptr, down = nullptr;  // copy streams of the pipelined host-state runs
  std::vector<cudaEvent_t> stage_ev;          // their chunk events
  CUtensorMap* tmaps = nullptr;         // TMA staging: two maps per (view, level) plane (tile box, source box)
  bool q_used = false;                  // a persistent launch was issued since the last check of its error word
  int nv = 0, nl = 0;
  ps_pm_params pm{};
  ps_filter_params fl{};
  uint64_t seed = 0;
  PsConsts cs{};
  std::vector<int> w, h;  // per (view, level)
  std::vector<int> nsrc;
  std::vector<std::vector<int>> sources;
  std::vector<PsLevel> lvh;  // host copies of the level and view tables
  std::vector<float> sweep_n;  // plane-sweep normal per view (3 floats; fronto-parallel by default)
  std::vector<PsView> vdh;
  // learned proposal buffers (network input / output of one view, grown on demand)
  unsigned short* netin = nullptr;
  size_t netin_cap = 0;
  float* netout = nullptr;
  size_t netout_cap = 0;
  unsigned long long* pcount = nullptr;
  FusedCloud fused;
  // device tables
  float* img = nullptr;
  PsLevel* lv = nullptr;
  PsPair* pairs = nullptr;
  PsLPair* lpairs = nullptr;
  PsView* views = nullptr;
  double* pairs64 = nullptr;
  int* has64 = nullptr;
  std::vector<Slot> slots;
  // snapshot
  float* snap = nullptr;
  size_t snap_cap = 0;
  long long* snap_off = nullptr;
  int snap_level = -1;
  bool snap_valid = false;
  uint64_t snap_id = 0;
  // pinned staging
  void* pin = nullptr;
  size_t pin_cap = 0;
  uint64_t launches = 0;
  size_t img_bytes = 0;
  std::vector<cudaArray_t> arrays;       // texture arrays (PS_TUNE_TEX_GATHER)
  std::vector<ps_backend::CachedArray> array_keys;  // their sizes and formats, handed back to the backend at the end
  std::vector<cudaTextureObject_t> texs;
  unsigned tuning = 0;
  // profiling
  bool profiling = false;
  unsigned long long* counters = nullptr;  // NCC windows per kernel kind, then PS_STAGE_STATS counters per kind
  struct Pending {
    int kind;
    cudaEvent_t a, b;
    bool persistent;  // owned by a captured graph (re-recorded on every replay)
  };
  std::vector<Pending> pending;
  double kind_ms[PS_KERNEL_KINDS] = {};
  uint64_t kind_launches[PS_KERNEL_KINDS] = {};
  bool capturing = false;  // a stream capture of this session's stream is in progress
  // captured single-level schedules (ps_schedule_resident)
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;  // captured schedule (nullptr: direct launches)
    long long* offsets = nullptr;    // snapshot offset table of the schedule's view set (device)
    uint64_t per_replay = 0;         // kernels per replay
    std::vector<Pending> events;     // per-launch event nodes captured with profiling on
    std::vector<long long*> level_offsets;  // multi-scale schedules: snapshot offset table per level (device)
  };
  std::map<std::string, GraphEntry> graphs;

  int W(int v, int l) const { return w[v * nl + l]; }
  int H(int v, int l) const { return h[v * nl + l]; }
};

namespace {

void fail(int code, const std::string& m) { throw PsError{code, m}; }
void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(e == cudaErrorMemoryAllocation ? PS_ENOMEM : PS_ECUDA,
         std::string("CUDA: ") + what + ": " + cudaGetErrorString(e));
  }
}

template <typename F>
int guard(ps_session* s, F&& f) {
  if (!s) return PS_EINVAL;
  try {
    cuda_ok(cudaSetDevice(s->be->device), "cudaSetDevice");
    f();
    s->err.clear();
    return PS_OK;
  } catch (const PsError& e) {
    s->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    s->err = "host allocation failed";
    return PS_ENOMEM;
  } catch (...) {
    s->err = "unexpected internal error";
    return PS_EINVAL;
  }
}

// An armed injected failure of `kind` (ps_backend_inject_failure): counts the operation down and fails it when the
// count is spent, before anything is issued to the device.
void maybe_inject(ps_session* s, uint32_t kind, const char* what) {
  ps_backend* be = s->be;
  if (!be || be->inject_kind != kind) return;
  if (be->inject_after > 0) {
    be->inject_after--;
    return;
  }
  be->inject_kind = PS_INJECT_NONE;
  fail(kind == PS_INJECT_DEVICE_ALLOC ? PS_ENOMEM : PS_ECUDA, std::string("injected failure: ") + what);
}

const char* site_name(unsigned site) {
  switch (site) {
    case PS_SITE_TILE: return "reference tile";
    case PS_SITE_BOX: return "staged source box";
    case PS_SITE_PLANE: return "source plane";
    case PS_SITE_STATE: return "state arrays";
    case PS_SITE_SOURCE: return "source view index";
    case PS_SITE_SNAPSHOT: return "depth snapshot";
    case PS_SITE_PROBE: return "self-test probe";
    default: return "unknown site";
  }
}

// Bounded waits (persistent queue, TMA barriers): after the stream has drained, a set error word (1 = queue, 2 = TMA)
// means a wait gave up; the word is cleared and the call fails with PS_ETIMEOUT.  An armed queue stall
// (PS_INJECT_QUEUE_STALL) is spent.
void check_queue(ps_session* s) {
  if (!s->q_used) return;
  s->q_used = false;
  if (s->be && s->be->inject_kind == PS_INJECT_QUEUE_STALL) s->be->inject_kind = PS_INJECT_NONE;
  unsigned e = 0;
  cuda_ok(cudaMemcpy(&e, s->qbuf + 1, sizeof e, cudaMemcpyDeviceToHost), "read queue error word");
  if (!e) return;
  cuda_ok(cudaMemset(s->qbuf + 1, 0, sizeof e), "clear queue error word");
  if (e == 3u) fail(PS_ECUDA, "staged half step: shared memory not aligned for TMA loads (nothing was loaded)");
  fail(PS_ETIMEOUT, e == 2u ? "staged half step: a wait for a TMA tile load gave up"
                            : "persistent half step: a wait for the previous half step's tiles gave up");
}

// Checked build: after the stream has drained, a non-zero fault word means a kernel skipped an out-of-bounds access.
// The word is cleared (so the session stays usable) and the call fails with PS_EFAULT naming the first violation.
// An armed self-test probe (PS_INJECT_CHECK_PROBE) is spent here.
void check_fault(ps_session* s) {
  if (!s->fault) return;
  unsigned long long w = 0;
  cuda_ok(cudaMemcpy(&w, s->fault, sizeof w, cudaMemcpyDeviceToHost), "read fault word");
  if (s->be && s->be->inject_kind == PS_INJECT_CHECK_PROBE) s->be->inject_kind = PS_INJECT_NONE;
  if (!w) return;
  cuda_ok(cudaMemset(s->fault, 0, sizeof w), "clear fault word");
  const unsigned site = (unsigned)(w >> 56);
  long long idx = (long long)(w & 0x00FFFFFFFFFFFFFFull);
  if (idx & 0x0080000000000000ll) idx -= 0x0100000000000000ll;  // sign of the 56-bit index
  fail(PS_EFAULT, std::string("checked build: out-of-bounds index ") + std::to_string(idx) + " (" + site_name(site) +
                      "); the access was skipped");
}

// Session device memory: from the backend's pool in the session stream's order (plain cudaMalloc when the device
// offers no pool).  Every use of a buffer is on the session stream.
template <typename T>
T* dalloc(ps_session* s, size_t n) {
  maybe_inject(s, PS_INJECT_DEVICE_ALLOC, "device allocation");
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  if (s->be && s->be->pool) cuda_ok(cudaMallocFromPoolAsync(&p, bytes, s->be->pool, s->st), "cudaMallocFromPoolAsync");
  else cuda_ok(cudaMalloc(&p, bytes), "cudaMalloc");
  return (T*)p;
}
void dfree(ps_session* s, void* p) {
  if (!p) return;
  if (s->be && s->be->pool) cudaFreeAsync(p, s->st);
  else cudaFree(p);
}

void* pinned(ps_session* s, size_t bytes) {
  if (bytes > s->pin_cap) {
    if (s->pin) cudaFreeHost(s->pin);
    s->pin = nullptr;
    s->pin_cap = 0;
    size_t cap = round_up(bytes + bytes / 4, 1 << 20);
    cuda_ok(cudaMallocHost(&s->pin, cap), "cudaMallocHost");
    s->pin_cap = cap;
  }
  return s->pin;
}

void check_views(ps_session* s, const uint32_t* views, size_t n) {
  if (n > 0 && !views) fail(PS_EINVAL, "views is NULL");
  for (size_t i = 0; i < n; ++i)
    if (views[i] >= (uint32_t)s->nv) fail(PS_EINVAL, "view index " + std::to_string(views[i]) + " out of range");
}

Slot& slot(ps_session* s, int level) {
  if (level < 0 || level >= s->nl) fail(PS_EINVAL, "level " + std::to_string(level) + " out of range");
  Slot& sl = s->slots[level];
  if (!sl.ready) {
    sl.off.assign(s->nv, 0);
    long long tot = 0;
    for (int v = 0; v < s->nv; ++v) {
      sl.off[v] = tot;
      tot += (long long)s->W(v, level) * s->H(v, level);
    }
    sl.total = tot;
    sl.plane = dalloc<float4>(s, tot);
    sl.aux = dalloc<float4>(s, tot);
    sl.prior = dalloc<float4>(s, tot);
    sl.cost = dalloc<float>(s, tot);
    sl.bview = dalloc<unsigned char>(s, tot);
    sl.count = dalloc<unsigned char>(s, tot);
    cuda_ok(cudaMemsetAsync(sl.plane, 0, std::max<long long>(tot, 1) * sizeof(float4), s->st), "memset");
    cuda_ok(cudaMemsetAsync(sl.bview, 255, std::max<long long>(tot, 1), s->st), "memset");
    sl.prior_valid.assign(s->nv, 0);
    sl.ready = true;
  }
  return sl;
}

// Splits a view list into launches of at most max_batch views and batch_pixels pixels (cf. Session::batches,
// crates/cuda/src/patchmatch.rs:607-625).
std::vector<std::pair<size_t, size_t>> batches(ps_session* s, const uint32_t* views, size_t n, int level) {
  std::vector<std::pair<size_t, size_t>> out;
  const size_t maxb = std::min<size_t>(s->be->opts.max_batch ? s->be->opts.max_batch : 64, PS_MAX_ITEMS);
  const uint64_t budget = s->be->opts.batch_pixels;
  size_t start = 0;
  uint64_t pix = 0;
  for (size_t i = 0; i < n; ++i) {
    uint64_t p = (uint64_t)s->W(views[i], level) * s->H(views[i], level);
    if (i > start && ((budget && pix + p > budget) || i - start >= maxb)) {
      out.push_back({start, i});
      start = i;
      pix = 0;
    }
    pix += p;
  }
  if (start < n) out.push_back({start, n});
  return out;
}

// TMA staging: two tensor maps per (view, level) plane over the session's image buffer (see tmap() in the kernels):
// map 0 with the reference tile's box (PS_HALF_ST_TW(wr) × PS_HALF_PH + 2·wr), map 1 with the source box
// (PS_BOX_P × PS_BOX_H).  The tensor is the whole bordered plane, pitch × (h + 2·PS_BORDER) f32 elements from its
// 128-byte aligned allocation; elements outside it read 0.
void build_tensor_maps(ps_session* s, const std::vector<PsLevel>& lvh, const std::vector<size_t>& offs,
                       const std::vector<size_t>& pitches) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      fail(PS_ECUDA, "cuTensorMapEncodeTiled is not available");
    encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  }
  const int wr = s->pm.window_radius;
  const cuuint32_t boxes[2][2] = {{(cuuint32_t)PS_HALF_ST_TW(wr), (cuuint32_t)(PS_HALF_PH + 2 * wr)},
                                  {(cuuint32_t)PS_BOX_P, (cuuint32_t)PS_BOX_H}};
  std::vector<CUtensorMap> maps(lvh.size() * 2);
  for (size_t i = 0; i < lvh.size(); ++i) {
    void* base = s->img + offs[i];
    if (((uintptr_t)base & 127u) || (pitches[i] * sizeof(float)) % 16) fail(PS_EINVAL, "plane not aligned for TMA");
    const cuuint64_t dims[2] = {(cuuint64_t)pitches[i], (cuuint64_t)(lvh[i].h + 2 * PS_BORDER)};
    const cuuint64_t strides[1] = {(cuuint64_t)(pitches[i] * sizeof(float))};
    const cuuint32_t es[2] = {1, 1};
    for (int k = 0; k < 2; ++k)
      if (encode(&maps[2 * i + k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, boxes[k], es,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        fail(PS_ECUDA, "cuTensorMapEncodeTiled failed");
  }
  s->tmaps = dalloc<CUtensorMap>(s, maps.size());
  cuda_ok(cudaMemcpyAsync(s->tmaps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, s->st),
          "upload tensor maps");
}

PsRun base_params(ps_session* s, int level) {
  PsRun P;
  memset(&P, 0, sizeof P);
  P.seed = s->seed;
  P.lv = s->lv;
  P.pairs = s->pairs;
  P.lpairs = s->lpairs;
  P.views = s->views;
  P.snap = s->snap;
  P.snap_off = s->snap_off;
  Slot& sl = slot(s, level);
  P.plane = sl.plane;
  P.cost = sl.cost;
  P.bview = sl.bview;
  P.count = sl.count;
  P.prior = sl.prior;
  P.nlevels = s->nl;
  P.level = level;
  P.topk = s->cs.topk;
  P.wr = s->pm.window_radius;
  P.ws = s->pm.window_step;
  P.tau_bad = s->cs.tau_bad;
  P.inv2beta2 = s->cs.inv2beta2;
  P.prev_w = s->cs.prev_w;
  P.n1 = s->cs.n1;
  P.n2 = s->cs.n2;
  P.inv2s = s->cs.inv2s;
  P.inv2c = s->cs.inv2c;
  P.cos_tri_min = s->cs.cos_tri_min;
  P.inv2inc = s->cs.inv2inc;
  P.lambda = s->cs.lambda;
  P.gmax = s->cs.gmax;
  P.cos_filter_tri = s->cs.cos_filter_tri;
  P.q_min = s->cs.q_min;
  P.ncc_norm = s->cs.ncc_norm;
  P.inv2ncc = s->cs.inv2ncc;
  P.filter_gmax = s->cs.filter_gmax;
  P.weak_var = s->cs.weak_var;
  P.need_min = (int)s->fl.min_num_consistent;
  P.fault = s->fault;
  P.state_pixels = sl.total;
  P.snap_pixels = (long long)s->snap_cap;
  P.nviews_all = s->nv;
  P.probe = s->fault && s->be && s->be->inject_kind == PS_INJECT_CHECK_PROBE && !s->capturing;
  P.queue = s->qbuf;  // word 1 is the error word of every bounded wait (queue, TMA)
  return P;
}

// Fills the item table for views[a..b) with tiles of pw × ph pixels; aux_level >= 0 stores that level's slot offset
// in item.aux.
void set_items(ps_session* s, PsRun& P, const uint32_t* views, size_t a, size_t b, int level, int pw, int ph,
               int aux_level = -1, const std::vector<long long>* aux_off = nullptr) {
  Slot& sl = s->slots[level];
  int tiles = 0, maxsrc = 1;
  P.nitems = (int)(b - a);
  for (size_t i = a; i < b; ++i) {
    const int v = (int)views[i];
    PsItem& it = P.items[i - a];
    it.view = v;
    it.w = s->W(v, level);
    it.h = s->H(v, level);
    it.off = sl.off[v];
    it.aux = aux_off ? (*aux_off)[v] : (aux_level >= 0 ? s->slots[aux_level].off[v] : 0);
    it.tile0 = tiles;
    tiles += ((it.w + pw - 1) / pw) * ((it.h + ph - 1) / ph);
    maxsrc = std::max(maxsrc, s->nsrc[v]);
  }
  P.ntiles = tiles;
  P.maxsrc = maxsrc;
}

void launched(ps_session* s, cudaError_t e, const char* what) {
  cuda_ok(e, what);
  s->launches++;
}

// Brackets one launch with CUDA events (profiling on) and points the NCC-window counter at its kind.
template <typename F>
void timed_launch(ps_session* s, int kind, PsRun& P, F&& f, const char* what) {
  if (!s->profiling) {
    P.ncc_count = nullptr;
    P.stage_count = nullptr;
    launched(s, f(P), what);
    return;
  }
  P.ncc_count = s->counters + kind;
  P.stage_count = s->counters + PS_KERNEL_KINDS + PS_STAGE_STATS * kind;
  ps_session::Pending pd;
  pd.kind = kind;
  pd.persistent = false;
  cuda_ok(cudaEventCreate(&pd.a), "cudaEventCreate");
  cuda_ok(cudaEventCreate(&pd.b), "cudaEventCreate");
  // inside a stream capture the records must be external event nodes (re-recorded on each replay), not the
  // capture-internal dependencies a plain cudaEventRecord expresses
  const unsigned flags = s->capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
  cuda_ok(cudaEventRecordWithFlags(pd.a, s->st, flags), "cudaEventRecord");
  launched(s, f(P), what);
  cuda_ok(cudaEventRecordWithFlags(pd.b, s->st, flags), "cudaEventRecord");
  s->pending.push_back(pd);
  s->kind_launches[kind]++;
}

// At least n copy events for the host-state transfers.
void xfer_events(ps_session* s, size_t n) {
  while (s->xfer.size() < n) {
    cudaEvent_t e;
    cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    s->xfer.push_back(e);
  }
}

void collect_events(ps_session* s) {
  if (s->pending.empty()) return;
  cuda_ok(cudaStreamSynchronize(s->st), "cudaStreamSynchronize");
  check_fault(s);
  check_queue(s);
  for (auto& pd : s->pending) {
    float ms = 0.f;
    cuda_ok(cudaEventElapsedTime(&ms, pd.a, pd.b), "cudaEventElapsedTime");
    s->kind_ms[pd.kind] += ms;
    if (!pd.persistent) {
      cudaEventDestroy(pd.a);
      cudaEventDestroy(pd.b);
    }
  }
  s->pending.clear();
}

void sync(ps_session* s) {
  cuda_ok(cudaStreamSynchronize(s->st), "cudaStreamSynchronize");
  check_fault(s);
  check_queue(s);
}

// Destroys every captured schedule graph: they hold device addresses of a buffer about to be replaced.
void drop_graphs(ps_session* s) {
  if (s->graphs.empty()) return;
  collect_events(s);  // finishes the stream and releases the replays' pending events
  for (auto& kv : s->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    dfree(s, kv.second.offsets);
    for (long long* o : kv.second.level_offsets) dfree(s, o);
    for (auto& pd : kv.second.events) {
      cudaEventDestroy(pd.a);
      cudaEventDestroy(pd.b);
    }
  }
  s->graphs.clear();
}

// Grows the snapshot buffer to `total` floats (captured graphs are dropped first).
void realloc_snapshot(ps_session* s, size_t total) {
  drop_graphs(s);
  if (s->snap) dfree(s, s->snap);
  s->snap = nullptr;
  s->snap_cap = 0;
  s->snap = dalloc<float>(s, std::max<size_t>(total, 1));
  s->snap_cap = total;
}

// ---- state packing (host) -------------------------------------------------------------------------------------
void check_state(ps_session* s, int v, int level, const ps_view_state& st) {
  if ((int)st.width != s->W(v, level) || (int)st.height != s->H(v, level))
    fail(PS_EINVAL, "state size " + std::to_string(st.width) + "x" + std::to_string(st.height) + " != level " +
                        std::to_string(s->W(v, level)) + "x" + std::to_string(s->H(v, level)));
}

// Uploads depth/normal (as planes) and optionally prior of views[a..b) into the level slot.
void upload_planes(ps_session* s, const uint32_t* views, size_t a, size_t b, const ps_view_state* states,
                   int level, bool with_prior, float4* dst_base = nullptr) {
  Slot& sl = slot(s, level);
  maybe_inject(s, PS_INJECT_UPLOAD, "upload states");
  size_t total = 0;
  for (size_t i = a; i < b; ++i) total += (size_t)states[i].width * states[i].height;
  float4* stage = (float4*)pinned(s, std::max<size_t>(total, 1) * sizeof(float4) * (with_prior ? 2 : 1));
  for (size_t i = a; i < b; ++i) {  // every view is checked before any copy is issued
    check_state(s, (int)views[i], level, states[i]);
    if (!states[i].depth || !states[i].normal) fail(PS_EINVAL, "state depth/normal is NULL");
  }
  size_t o = 0;
  float4* dst = dst_base ? dst_base : sl.plane;
  for (size_t i = a; i < b; ++i) {  // each view's copy starts as soon as it is packed, while the next view is packed
    const ps_view_state& st = states[i];
    const long long n = (long long)st.width * st.height;
    float4* q = stage + o;
#pragma omp parallel for schedule(static) if (n > 65536)
    for (long long p = 0; p < n; ++p) q[p] = make_float4(st.normal[3 * p], st.normal[3 * p + 1], st.normal[3 * p + 2], st.depth[p]);
    cuda_ok(cudaMemcpyAsync(dst + sl.off[views[i]], q, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice, s->st),
            "upload planes");
    o += (size_t)n;
  }
  if (with_prior) {
    float4* pst = stage + total;
    size_t po = 0;
    for (size_t i = a; i < b; ++i) {
      const ps_view_state& st = states[i];
      const size_t n = (size_t)st.width * st.height;
      if (st.prior) {
        memcpy(pst + po, st.prior, n * sizeof(float4));
        cuda_ok(cudaMemcpyAsync(sl.prior + sl.off[views[i]], pst + po, n * sizeof(float4), cudaMemcpyHostToDevice,
                                s->st),
                "upload prior");
        sl.prior_valid[views[i]] = 1;
      } else {
        sl.prior_valid[views[i]] = 0;
      }
      po += n;
    }
  }
  sync(s);  // the staging buffer is reused by the next call
}

// Downloads planes (from `src` or the slot planes) and/or costs into host states.
void download_states(ps_session* s, const uint32_t* views, size_t a, size_t b, ps_view_state* states, int level,
                     bool planes, bool costs, const float4* src = nullptr) {
  Slot& sl = slot(s, level);
  size_t total = 0;
  for (size_t i = a; i < b; ++i) total += (size_t)s->W(views[i], level) * s->H(views[i], level);
  float4* stage = (float4*)pinned(s, std::max<size_t>(total, 1) * (sizeof(float4) + sizeof(float)));
  float* cst = (float*)(stage + total);
  for (size_t i = a; i < b; ++i) {  // every view is checked before any copy is issued
    check_state(s, (int)views[i], level, states[i]);
    if (planes && (!states[i].depth || !states[i].normal)) fail(PS_EINVAL, "state depth/normal is NULL");
    if (costs && !states[i].cost) fail(PS_EINVAL, "state cost is NULL");
  }
  size_t o = 0;
  std::vector<size_t> so;
  xfer_events(s, b - a);
  for (size_t i = a; i < b; ++i) {
    const int v = (int)views[i];
    const size_t n = (size_t)s->W(v, level) * s->H(v, level);
    so.push_back(o);
    if (planes)
      cuda_ok(cudaMemcpyAsync(stage + o, (src ? src : sl.plane) + sl.off[v], n * sizeof(float4),
                              cudaMemcpyDeviceToHost, s->st),
              "download planes");
    if (costs)
      cuda_ok(cudaMemcpyAsync(cst + o, sl.cost + sl.off[v], n * sizeof(float), cudaMemcpyDeviceToHost, s->st),
              "download cost");
    cuda_ok(cudaEventRecord(s->xfer[i - a], s->st), "cudaEventRecord");
    o += n;
  }
  // each view is unpacked as soon as its own copies are done, while the later views' copies run
  for (size_t i = a; i < b; ++i) {
    cuda_ok(cudaEventSynchronize(s->xfer[i - a]), "cudaEventSynchronize");
    ps_view_state& st = states[i];
    const long long n = (long long)st.width * st.height;
    const float4* q = stage + so[i - a];
    if (planes) {
#pragma omp parallel for schedule(static) if (n > 65536)
      for (long long p = 0; p < n; ++p) {
        st.normal[3 * p] = q[p].x;
        st.normal[3 * p + 1] = q[p].y;
        st.normal[3 * p + 2] = q[p].z;
        st.depth[p] = q[p].w;
      }
    }
    if (costs) {
      memcpy(st.cost, cst + so[i - a], n * sizeof(float));
    }
  }
  sync(s);  // fault and error words
}

// Uploads a host snapshot (re-uploaded only when its id or level changes, cf. Session::ensure_snapshot,
// crates/cuda/src/patchmatch.rs:573-604).
void ensure_snapshot(ps_session* s, const ps_depth_snapshot* snap) {
  if (!snap) fail(PS_EINVAL, "a geometric run needs a snapshot");
  if (snap->level >= (uint32_t)s->nl) fail(PS_EINVAL, "snapshot level out of range");
  if (s->snap_valid && s->snap_id == snap->id && s->snap_level == (int)snap->level) return;
  const int l = (int)snap->level;
  std::vector<long long> offs(s->nv, -1);
  size_t total = 0;
  for (int v = 0; v < s->nv; ++v) {
    const uint64_t need = (uint64_t)s->W(v, l) * s->H(v, l);
    if ((uint32_t)v < snap->num_maps && snap->maps && snap->maps[v] &&
        (!snap->map_lengths || snap->map_lengths[v] == need)) {
      offs[v] = (long long)total;
      total += (size_t)need;
    }
  }
  maybe_inject(s, PS_INJECT_UPLOAD, "upload snapshot");
  if (total > s->snap_cap) {
    realloc_snapshot(s, total);
  }
  for (int v = 0; v < s->nv; ++v)
    if (offs[v] >= 0)
      cuda_ok(cudaMemcpyAsync(s->snap + offs[v], snap->maps[v], (size_t)s->W(v, l) * s->H(v, l) * sizeof(float),
                              cudaMemcpyHostToDevice, s->st),
              "upload snapshot");
  cuda_ok(cudaMemcpyAsync(s->snap_off, offs.data(), s->nv * sizeof(long long), cudaMemcpyHostToDevice, s->st),
          "upload snapshot offsets");
  sync(s);
  s->snap_valid = true;
  s->snap_id = snap->id;
  s->snap_level = l;
}

// Eval (mode 1) + iterations × two colours on the resident slot of views[a..b).
void run_batch(ps_session* s, const uint32_t* views, size_t a, size_t b, const ps_run_params* p, bool use_prior) {
  PsRun P = base_params(s, (int)p->level);
  P.geometric = p->geometric ? 1 : 0;
  P.run_id = (int)p->run_id;
  P.random_init = p->random_init ? 1 : 0;
  P.use_prior = use_prior ? 1 : 0;
  P.mode = 1;
  if (p->random_init == PS_INIT_PROPOSAL) {
    Slot& sl = s->slots[p->level];
    for (size_t i = a; i < b; ++i)
      if (!sl.proposal || !sl.proposal_valid[views[i]])
        fail(PS_EINVAL, "view " + std::to_string(views[i]) + " has no proposal at level " + std::to_string(p->level));
    P.proposal = sl.proposal;
  }
  set_items(s, P, views, a, b, (int)p->level, PS_EVAL_PW, PS_EVAL_PH);
  timed_launch(s, PS_KERNEL_EVAL, P, [&](const PsRun& q) { return s->L->eval(q, s->tuning & PS_TUNE_TEX_GATHER, s->st); }, "evaluate kernel");
  PsRun H = P;
  set_items(s, H, views, a, b, (int)p->level, s->L->half_lanes(s->tuning) == 2 ? PS_HALF2_PW : PS_HALF_PW,
            PS_HALF_PH);
  if (s->L->half_run_ok(s->tuning, H.wr, H.ws)) {
    // persistent kernel: up to PS_MAX_PHASES half steps per launch, over a zeroed queue
    for (uint32_t t0 = 0; t0 < p->iterations; t0 += PS_MAX_PHASES / 2) {
      const uint32_t n = std::min<uint32_t>(p->iterations - t0, PS_MAX_PHASES / 2);
      H.nphases = (int)(2 * n);
      for (uint32_t k = 0; k < 2 * n; ++k) {
        PsPhase& q = H.phases[k];
        q.t = (int)(t0 + k / 2);
        q.color = (int)(k & 1);
        ps_iter_consts(&s->pm, P.geometric, q.t, &q.tau_good, &q.eps, &q.phi);
      }
      H.queue = s->qbuf;
      H.qstall = s->be && s->be->inject_kind == PS_INJECT_QUEUE_STALL && !s->capturing;
      // the queue counter and the done counts; the error word (qbuf[1]) keeps what earlier launches set
      cuda_ok(cudaMemsetAsync(s->qbuf, 0, sizeof(unsigned), s->st), "memset queue");
      cuda_ok(cudaMemsetAsync(s->qbuf + 2, 0, (size_t)H.nphases * H.nitems * sizeof(unsigned), s->st),
              "memset queue");
      timed_launch(s, PS_KERNEL_HALF, H, [&](const PsRun& q) { return s->L->half_run(q, s->tuning, s->st); },
                   "persistent half-step kernel");
      s->q_used = true;
    }
    return;
  }
  H.tmaps = s->tmaps;
  if (s->tmaps) s->q_used = true;  // the TMA waits report through the error word
  for (uint32_t t = 0; t < p->iterations; ++t) {
    H.t = (int)t;
    ps_iter_consts(&s->pm, P.geometric, (int)t, &H.tau_good, &H.eps, &H.phi);
    for (int color = 0; color < 2; ++color) {
      H.color = color;
      timed_launch(s, PS_KERNEL_HALF, H, [&](const PsRun& q) { return s->L->half(q, s->tuning, s->st); },
                   "half-step kernel");
    }
  }
}

void require_snapshot_level(ps_session* s, int level) {
  if (!s->snap_valid) fail(PS_EINVAL, "a geometric run needs a snapshot");
  if (s->snap_level != level) fail(PS_EINVAL, "snapshot level differs from the run level");
}

}  // namespace

// ================================================================================================ C ABI
extern "C" {

int ps_abi_version(void) { return PS_ABI_VERSION; }
void ps_pm_params_default(ps_pm_params* out) {
  if (out) ps_default_pm(out);
}
void ps_filter_params_default(ps_filter_params* out) {
  if (out) ps_default_filter(out);
}
void ps_options_default(ps_options* out) {
  if (!out) return;
  memset(out, 0, sizeof *out);
  out->math_mode = PS_MATH_PARITY;
  out->max_batch = 64;
  out->batch_pixels = 0;
}

int ps_backend_create(int device, const ps_options* opts, ps_backend** out) {
  if (!out) return PS_EINVAL;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return PS_ENODEV;
  }
  if (device < 0 || device >= n) return PS_ENODEV;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PS_ENODEV;
  if (prop.major != 10) return PS_ENODEV;  // the kernels are built for sm_100a only
  ps_backend* be = new (std::nothrow) ps_backend();
  if (!be) return PS_ENOMEM;
  be->device = device;
  ps_options_default(&be->opts);
  if (opts) be->opts = *opts;
  if (be->opts.math_mode > PS_MATH_FAST || be->opts.checked > 1 ||
      (be->opts.checked && be->opts.math_mode == PS_MATH_FAST) || (be->opts.tuning & ~PS_TUNE_VALID_MASK)) {
    delete be;
    return PS_EINVAL;
  }
  be->name = std::string("b200(") + prop.name +
             (be->opts.checked ? ", parity, checked)" : be->opts.math_mode == PS_MATH_FAST ? ", fast)" : ", parity)");
  cudaMemPoolProps pp;
  memset(&pp, 0, sizeof pp);
  pp.allocType = cudaMemAllocationTypePinned;
  pp.handleTypes = cudaMemHandleTypeNone;
  pp.location.type = cudaMemLocationTypeDevice;
  pp.location.id = device;
  if (cudaMemPoolCreate(&be->pool, &pp) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;  // keep freed memory in the pool until the backend is destroyed
    if (cudaMemPoolSetAttribute(be->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
      cudaMemPoolDestroy(be->pool);
      be->pool = nullptr;
    }
  } else {
    be->pool = nullptr;
  }
  cudaGetLastError();
  *out = be;
  return PS_OK;
}

void ps_backend_destroy(ps_backend* be) {
  if (!be) return;
  cudaSetDevice(be->device);
  if (be->pin) cudaFreeHost(be->pin);
  for (auto& c : be->arrays) cudaFreeArray(c.a);
  if (be->pool) cudaMemPoolDestroy(be->pool);
  cudaGetLastError();
  delete be;
}
const char* ps_backend_name(const ps_backend* be) { return be ? be->name.c_str() : ""; }
const char* ps_backend_last_error(const ps_backend* be) { return be ? be->err.c_str() : "backend is NULL"; }
const char* ps_last_error(const ps_session* s) { return s ? s->err.c_str() : "session is NULL"; }
uint64_t ps_launch_count(const ps_session* s) { return s ? s->launches : 0; }

int ps_backend_inject_failure(ps_backend* be, uint32_t kind, uint32_t after) {
  if (!be || kind > PS_INJECT_QUEUE_STALL) return PS_EINVAL;
  if (kind == PS_INJECT_CHECK_PROBE && !be->opts.checked) return PS_EINVAL;
  std::lock_guard<std::mutex> g(be->mu);
  be->inject_kind = kind;
  be->inject_after = after;
  return PS_OK;
}

int ps_begin(ps_backend* be, const ps_kernel_input* in, ps_session** out) {
  if (!be || !in || !out) return PS_EINVAL;
  *out = nullptr;
  {
    std::lock_guard<std::mutex> g(be->mu);
    if (be->busy) {
      be->err = "the backend already has an open session";
      return PS_EBUSY;
    }
    be->busy = true;
  }
  ps_session* s = new (std::nothrow) ps_session();
  if (!s) {
    std::lock_guard<std::mutex> g(be->mu);
    be->busy = false;
    return PS_ENOMEM;
  }
  s->be = be;
  s->pin = be->pin;  // pinned staging kept from the backend's previous session
  s->pin_cap = be->pin_cap;
  be->pin = nullptr;
  be->pin_cap = 0;
  int rc = guard(s, [&] {
    const ps_pm_params& pm = in->pm;
    if (pm.window_radius < 1 || pm.window_radius > 20 || pm.window_step < 1 || pm.window_step > 2)
      fail(PS_EINVAL, "window radius " + std::to_string(pm.window_radius) + " (1..=20), step " +
                          std::to_string(pm.window_step) + " (1|2)");
    if (in->num_levels < 1) fail(PS_EINVAL, "num_levels must be >= 1");
    if (in->num_views > 0 && !in->views) fail(PS_EINVAL, "views is NULL");
    s->nv = (int)in->num_views;
    s->nl = (int)in->num_levels;
    s->pm = pm;
    s->fl = in->filter;
    s->seed = in->seed;
    s->cs = ps_session_consts(&s->pm, &s->fl);
    s->L = be->opts.checked ? &kChecked : (be->opts.math_mode == PS_MATH_FAST ? &kFast : &kParity);
    s->tuning = be->opts.tuning;
    s->w.assign(s->nv * s->nl, 0);
    s->h.assign(s->nv * s->nl, 0);
    s->nsrc.assign(s->nv, 0);
    s->sources.assign(s->nv, {});
    // validation (crates/cuda/src/patchmatch.rs:292-294, :366-371)
    size_t total = 0;
    std::vector<size_t> offs(s->nv * s->nl), pitches(s->nv * s->nl);
    for (int v = 0; v < s->nv; ++v) {
      const ps_kernel_view& kv = in->views[v];
      if (!kv.levels) fail(PS_EINVAL, "view " + std::to_string(v) + ": levels is NULL");
      if (kv.num_sources > PS_MAX_SOURCES)
        fail(PS_EINVAL, "view " + std::to_string(v) + ": " + std::to_string(kv.num_sources) + " sources > 32");
      if (kv.num_sources > 0 && (!kv.sources || !kv.pairs))
        fail(PS_EINVAL, "view " + std::to_string(v) + ": sources/pairs is NULL");
      for (uint32_t j = 0; j < kv.num_sources; ++j)
        if (kv.sources[j] >= in->num_views) fail(PS_EINVAL, "view " + std::to_string(v) + ": source out of range");
      s->nsrc[v] = (int)kv.num_sources;
      s->sources[v].assign(kv.sources, kv.sources + kv.num_sources);
      for (int l = 0; l < s->nl; ++l) {
        const ps_level_image& li = kv.levels[l];
        if (li.width < 1 || li.height < 1 || !li.pixels || li.format > PS_IMAGE_F32)
          fail(PS_EINVAL, "view " + std::to_string(v) + " level " + std::to_string(l) + ": bad image");
        if (li.width > (1u << 15) || li.height > (1u << 15)) fail(PS_EINVAL, "image larger than 32768 pixels");
        if (!(li.k[0] != 0.0f) || !(li.k[1] != 0.0f)) fail(PS_EINVAL, "focal length is zero");
        s->w[v * s->nl + l] = (int)li.width;
        s->h[v * s->nl + l] = (int)li.height;
        const size_t pitch = round_up(li.width + 2 * PS_BORDER, 32);
        total = round_up(total, 32);
        offs[v * s->nl + l] = total;
        pitches[v * s->nl + l] = pitch;
        total += pitch * (li.height + 2 * PS_BORDER);
      }
    }
    cuda_ok(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking), "cudaStreamCreate");
    // module constants are set here, outside any stream capture (their copy is synchronous)
    cuda_ok(ps_parity::prepare(), "module constants");
    cuda_ok(ps_fast::prepare(), "module constants");
    s->qbuf = dalloc<unsigned>(s, 2 + (size_t)PS_MAX_PHASES * PS_MAX_ITEMS);
    if (be->opts.checked) {
      cuda_ok(ps_checked::prepare(), "module constants");
      s->fault = dalloc<unsigned long long>(s, 1);
      cuda_ok(cudaMemsetAsync(s->fault, 0, sizeof(unsigned long long), s->st), "memset");
    }
    // images: normalised f32 planes with a zero border.  8-bit images travel as bytes through the pinned staging
    // buffer and are expanded on the device with a table of the correctly rounded u/255 (the oracle's plane values);
    // f32 images are copied row by row into the bordered plane.
    std::vector<PsLevel> lvh(s->nv * s->nl);
    s->img = dalloc<float>(s, total);
    s->img_bytes = total * sizeof(float);
    cuda_ok(cudaMemsetAsync(s->img, 0, std::max<size_t>(total, 1) * sizeof(float), s->st), "memset images");
    size_t u8_total = 0;
    std::vector<size_t> u8_off(s->nv * s->nl, 0);
    for (int v = 0; v < s->nv; ++v)
      for (int l = 0; l < s->nl; ++l) {
        const ps_level_image& li = in->views[v].levels[l];
        if (li.format != PS_IMAGE_U8) continue;
        u8_off[v * s->nl + l] = u8_total;
        u8_total += round_up((size_t)li.width * li.height, 16);
      }
    unsigned char* d8 = nullptr;  // the 8-bit images on the device, then the table
    if (u8_total) {
      unsigned char* stage = (unsigned char*)pinned(s, u8_total + 256 * sizeof(float));
      float* lut = (float*)(stage + u8_total);
      for (int u = 0; u < 256; ++u) lut[u] = ps_u8_unit((unsigned char)u);
      std::vector<std::pair<int, int>> u8_images;
      for (int v = 0; v < s->nv; ++v)
        for (int l = 0; l < s->nl; ++l)
          if (in->views[v].levels[l].format == PS_IMAGE_U8) u8_images.push_back({v, l});
#pragma omp parallel for schedule(dynamic)
      for (long long k = 0; k < (long long)u8_images.size(); ++k) {
        const ps_level_image& li = in->views[u8_images[k].first].levels[u8_images[k].second];
        unsigned char* dst = stage + u8_off[u8_images[k].first * s->nl + u8_images[k].second];
        const size_t stride = li.stride ? li.stride : li.width;
        for (uint32_t y = 0; y < li.height; ++y)
          memcpy(dst + (size_t)y * li.width, (const unsigned char*)li.pixels + y * stride, li.width);
      }
      d8 = dalloc<unsigned char>(s, u8_total + 256 * sizeof(float));
      maybe_inject(s, PS_INJECT_UPLOAD, "upload 8-bit images");
      cuda_ok(cudaMemcpyAsync(d8, stage, u8_total + 256 * sizeof(float), cudaMemcpyHostToDevice, s->st),
              "upload 8-bit images");
    }
    for (int v = 0; v < s->nv; ++v)
      for (int l = 0; l < s->nl; ++l) {
        const ps_level_image& li = in->views[v].levels[l];
        const size_t pitch = pitches[v * s->nl + l];
        float* dst = s->img + offs[v * s->nl + l] + PS_BORDER * pitch + PS_BORDER;
        if (li.format == PS_IMAGE_U8) {
          launched(s,
                   ps_post::launch_u8_plane(d8 + u8_off[v * s->nl + l], (int)li.width, (int)li.height,
                                            (const float*)(d8 + u8_total), dst, (int)pitch, s->st),
                   "image plane kernel");
        } else {
          const size_t stride = li.stride ? li.stride : li.width;
          maybe_inject(s, PS_INJECT_UPLOAD, "upload image");
          cuda_ok(cudaMemcpy2DAsync(dst, pitch * sizeof(float), li.pixels, stride * sizeof(float),
                                    li.width * sizeof(float), li.height, cudaMemcpyHostToDevice, s->st),
                  "upload image");
        }
        PsLevel& L = lvh[v * s->nl + l];
        L.img = dst;
        L.tex = 0;
        L.w = (int)li.width;
        L.h = (int)li.height;
        L.pitch = (int)pitch;
        L.pad = 0;
        L.fx = li.k[0];
        L.fy = li.k[1];
        L.cx = li.k[2];
        L.cy = li.k[3];
      }
    if (s->tuning & PS_TUNE_TEX_GATHER) {
      // one gather-capable CUDA array + border-addressed point texture per (view, level).  8-bit images keep 8-bit
      // texels read as normalized floats (the texture unit returns the correctly rounded u/255, the plane's value, for
      // every u); f32 images are copied from the plane.
      const cudaChannelFormatDesc cdf = cudaCreateChannelDesc<float>();
      const cudaChannelFormatDesc cd8 = cudaCreateChannelDesc<unsigned char>();
      for (int v = 0; v < s->nv; ++v)
        for (int l = 0; l < s->nl; ++l) {
          PsLevel& L = lvh[v * s->nl + l];
          const ps_level_image& li = in->views[v].levels[l];
          const bool u8 = li.format == PS_IMAGE_U8;
          cudaArray_t arr = nullptr;
          auto& cache = be->arrays;
          for (size_t k = 0; k < cache.size(); ++k)
            if (cache[k].w == L.w && cache[k].h == L.h && cache[k].u8 == u8) {
              arr = cache[k].a;
              cache.erase(cache.begin() + (long)k);
              break;
            }
          if (!arr)
            cuda_ok(cudaMallocArray(&arr, u8 ? &cd8 : &cdf, L.w, L.h, cudaArrayTextureGather), "cudaMallocArray");
          s->arrays.push_back(arr);
          s->array_keys.push_back({arr, L.w, L.h, u8});
          if (u8)
            cuda_ok(cudaMemcpy2DToArrayAsync(arr, 0, 0, d8 + u8_off[v * s->nl + l], L.w, L.w, L.h,
                                             cudaMemcpyDeviceToDevice, s->st),
                    "copy texture array");
          else
            cuda_ok(cudaMemcpy2DToArrayAsync(arr, 0, 0, L.img, L.pitch * sizeof(float), L.w * sizeof(float), L.h,
                                             cudaMemcpyDeviceToDevice, s->st),
                    "copy texture array");
          cudaResourceDesc rd;
          memset(&rd, 0, sizeof rd);
          rd.resType = cudaResourceTypeArray;
          rd.res.array.array = arr;
          cudaTextureDesc td;
          memset(&td, 0, sizeof td);
          td.addressMode[0] = td.addressMode[1] = cudaAddressModeBorder;
          td.filterMode = cudaFilterModePoint;
          td.readMode = u8 ? cudaReadModeNormalizedFloat : cudaReadModeElementType;
          td.normalizedCoords = 0;
          cudaTextureObject_t t = 0;
          cuda_ok(cudaCreateTextureObject(&t, &rd, &td, nullptr), "cudaCreateTextureObject");
          s->texs.push_back(t);
          L.tex = (unsigned long long)t;
        }
    }
    if (d8) {
      sync(s);  // the pinned staging buffer is reused by the next call
      dfree(s, d8);
    }
    s->counters = dalloc<unsigned long long>(s, (1 + PS_STAGE_STATS) * PS_KERNEL_KINDS);
    cuda_ok(cudaMemsetAsync(s->counters, 0, (1 + PS_STAGE_STATS) * PS_KERNEL_KINDS * sizeof(unsigned long long), s->st), "memset");
    s->lvh = lvh;
    if ((s->tuning & PS_TUNE_TMA) && (s->tuning & PS_TUNE_STAGED)) build_tensor_maps(s, lvh, offs, pitches);
    s->lv = dalloc<PsLevel>(s, lvh.size());
    cuda_ok(cudaMemcpyAsync(s->lv, lvh.data(), lvh.size() * sizeof(PsLevel), cudaMemcpyHostToDevice, s->st), "upload levels");
    // pairs, views, FP64 pair tables
    std::vector<PsPair> prh((size_t)std::max(s->nv, 1) * PS_MAXSRC);
    std::vector<double> p64((size_t)std::max(s->nv, 1) * PS_MAXSRC * 15, 0.0);
    std::vector<int> has64(std::max(s->nv, 1), 0);
    std::vector<PsView> vdh(std::max(s->nv, 1));
    for (auto& p : prh) {
      memset(&p, 0, sizeof p);
      p.src = -1;
    }
    for (int v = 0; v < s->nv; ++v) {
      const ps_kernel_view& kv = in->views[v];
      for (uint32_t j = 0; j < kv.num_sources; ++j) {
        PsPair& p = prh[v * PS_MAXSRC + j];
        memcpy(p.r, kv.pairs[j].r, sizeof p.r);
        memcpy(p.t, kv.pairs[j].t, sizeof p.t);
        memcpy(p.c, kv.pairs[j].center, sizeof p.c);
        p.src = (int)kv.sources[j];
        if (kv.pairs_f64) memcpy(&p64[((size_t)v * PS_MAXSRC + j) * 15], kv.pairs_f64 + (size_t)j * 15, 15 * sizeof(double));
      }
      has64[v] = kv.pairs_f64 ? 1 : 0;
      vdh[v].key = kv.key;
      vdh[v].dmin = kv.depth_min;
      vdh[v].dmax = kv.depth_max;
      vdh[v].nsrc = (int)kv.num_sources;
      vdh[v].pad = 0;
    }
    s->vdh = vdh;
    s->sweep_n.assign(3 * (size_t)std::max(s->nv, 1), 0.0f);
    for (int v = 0; v < s->nv; ++v) s->sweep_n[3 * v + 2] = -1.0f;
    s->pairs = dalloc<PsPair>(s, prh.size());
    s->views = dalloc<PsView>(s, vdh.size());
    s->pairs64 = dalloc<double>(s, p64.size());
    s->has64 = dalloc<int>(s, has64.size());
    s->lpairs = dalloc<PsLPair>(s, (size_t)std::max(s->nv, 1) * s->nl * PS_MAXSRC);
    cuda_ok(cudaMemcpyAsync(s->pairs, prh.data(), prh.size() * sizeof(PsPair), cudaMemcpyHostToDevice, s->st), "upload pairs");
    cuda_ok(cudaMemcpyAsync(s->views, vdh.data(), vdh.size() * sizeof(PsView), cudaMemcpyHostToDevice, s->st), "upload views");
    cuda_ok(cudaMemcpyAsync(s->pairs64, p64.data(), p64.size() * sizeof(double), cudaMemcpyHostToDevice, s->st), "upload pairs64");
    cuda_ok(cudaMemcpyAsync(s->has64, has64.data(), has64.size() * sizeof(int), cudaMemcpyHostToDevice, s->st), "upload has64");
    launched(s, ps_parity::launch_setup_lpairs(s->lv, s->pairs, s->pairs64, s->has64, s->lpairs, s->nv, s->nl, s->st),
             "homography setup kernel");
    s->snap_off = dalloc<long long>(s, std::max(s->nv, 1));
    std::vector<long long> none(std::max(s->nv, 1), -1);
    cuda_ok(cudaMemcpyAsync(s->snap_off, none.data(), none.size() * sizeof(long long), cudaMemcpyHostToDevice, s->st), "upload");
    s->snap = dalloc<float>(s, 1);
    s->snap_cap = 1;
    s->slots.assign(s->nl, Slot());
    sync(s);
  });
  if (rc != PS_OK) {
    be->err = s->err;
    ps_end(s);
    return rc;
  }
  *out = s;
  return PS_OK;
}

int ps_end(ps_session* s) {
  if (!s) return PS_EINVAL;
  if (s->be) cudaSetDevice(s->be->device);
  if (s->st) cudaStreamSynchronize(s->st);
  for (Slot& sl : s->slots) {
    dfree(s, sl.plane);
    dfree(s, sl.aux);
    dfree(s, sl.prior);
    dfree(s, sl.cost);
    dfree(s, sl.bview);
    dfree(s, sl.count);
    dfree(s, sl.proposal);
    dfree(s, sl.pconf);
    dfree(s, sl.spk);
    dfree(s, sl.marks);
    dfree(s, sl.consumed);
    dfree(s, sl.cinit);
  }
  s->fused.release([s](void* q) { dfree(s, q); });
  dfree(s, s->fused.counter);
  dfree(s, s->fused.views);
  dfree(s, s->netin);
  dfree(s, s->netout);
  dfree(s, s->pcount);
  dfree(s, s->img);
  dfree(s, s->lv);
  dfree(s, s->pairs);
  dfree(s, s->lpairs);
  dfree(s, s->views);
  dfree(s, s->pairs64);
  dfree(s, s->has64);
  dfree(s, s->snap);
  dfree(s, s->snap_off);
  dfree(s, s->qbuf);
  dfree(s, s->tmaps);
  for (cudaEvent_t e : s->xfer) cudaEventDestroy(e);
  dfree(s, s->fault);
  for (cudaTextureObject_t t : s->texs) cudaDestroyTextureObject(t);
  if (s->be) {  // arrays no session reused are freed; this session's arrays wait for the next one
    for (auto& c : s->be->arrays) cudaFreeArray(c.a);
    s->be->arrays = s->array_keys;
  } else {
    for (cudaArray_t a : s->arrays) cudaFreeArray(a);
  }
  dfree(s, s->counters);
  for (auto& pd : s->pending) {
    if (pd.persistent) continue;  // destroyed with their graph below
    cudaEventDestroy(pd.a);
    cudaEventDestroy(pd.b);
  }
  for (auto& kv : s->graphs) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    dfree(s, kv.second.offsets);
    for (long long* o : kv.second.level_offsets) dfree(s, o);
    for (auto& pd : kv.second.events) {
      cudaEventDestroy(pd.a);
      cudaEventDestroy(pd.b);
    }
  }
  if (s->st) cudaStreamSynchronize(s->st);  // the frees above are stream-ordered
  if (s->be && s->pin) {
    if (s->be->pin) cudaFreeHost(s->be->pin);
    s->be->pin = s->pin;  // the pinned staging buffer stays with the backend for its next session
    s->be->pin_cap = s->pin_cap;
  } else if (s->pin) {
    cudaFreeHost(s->pin);
  }
  if (s->up) cudaStreamSynchronize(s->up);
  if (s->down) cudaStreamSynchronize(s->down);
  if (s->st) cudaStreamDestroy(s->st);
  if (s->up) cudaStreamDestroy(s->up);
  if (s->down) cudaStreamDestroy(s->down);
  for (cudaEvent_t e : s->stage_ev) cudaEventDestroy(e);
  cudaGetLastError();
  if (s->be) {
    std::lock_guard<std::mutex> g(s->be->mu);
    s->be->busy = false;
  }
  delete s;
  return PS_OK;
}

int ps_state_upload(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_view_state* states) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (n && !states) fail(PS_EINVAL, "states is NULL");
    upload_planes(s, views, 0, n, states, (int)level, true);
    Slot& sl = slot(s, (int)level);
    // costs too
    for (size_t i = 0; i < n; ++i)
      if (states[i].cost)
        cuda_ok(cudaMemcpyAsync(sl.cost + sl.off[views[i]], states[i].cost,
                                (size_t)states[i].width * states[i].height * sizeof(float), cudaMemcpyHostToDevice, s->st),
                "upload cost");
    sync(s);
  });
}

int ps_state_download(ps_session* s, uint32_t level, const uint32_t* views, size_t n, ps_view_state* states) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (n && !states) fail(PS_EINVAL, "states is NULL");
    download_states(s, views, 0, n, states, (int)level, true, true);
  });
}

int ps_run_resident(ps_session* s, const uint32_t* views, size_t n, const ps_run_params* p) {
  return guard(s, [&] {
    if (!p) fail(PS_EINVAL, "params is NULL");
    if (p->random_init > PS_INIT_PROPOSAL) fail(PS_EINVAL, "random_init must be 0, 1 or 2");
    check_views(s, views, n);
    Slot& sl = slot(s, (int)p->level);
    if (p->geometric) require_snapshot_level(s, (int)p->level);
    for (auto [a, b] : batches(s, views, n, (int)p->level)) {
      bool up = p->use_prior != 0;
      for (size_t i = a; i < b; ++i) up = up && sl.prior_valid[views[i]];
      run_batch(s, views, a, b, p, up);
    }
  });
}

namespace {
// Host-state runs of at least this many pixels are pipelined (run_pipelined); smaller ones gain nothing from it.
constexpr size_t kPipelinePixels = size_t(1) << 22;

// A photometric or geometric run of views[a, b) with host states, pipelined: the views go in up to three chunks of
// about equal pixel count, and while chunk k runs on the session stream, chunk k + 1's states are packed on the host
// and copied in on one copy stream, and chunk k - 1's results are copied out on the other and unpacked.  Views are
// independent within a run, so the chunks compute exactly what one launch over all of them computes.
void run_pipelined(ps_session* s, const uint32_t* views, size_t a, size_t b, ps_view_state* states,
                   const ps_run_params* p) {
  const int level = (int)p->level;
  Slot& sl = slot(s, level);
  const bool upload = !p->random_init;
  std::vector<size_t> px(b - a);
  size_t total = 0;
  for (size_t i = a; i < b; ++i) {
    check_state(s, (int)views[i], level, states[i]);
    if (!states[i].depth || !states[i].normal || !states[i].cost) fail(PS_EINVAL, "state depth/normal/cost is NULL");
    px[i - a] = (size_t)states[i].width * states[i].height;
    total += px[i - a];
  }
  // chunk boundaries by pixel count
  std::vector<size_t> cut{a};
  const int K = (int)std::min<size_t>(3, b - a);
  size_t acc = 0;
  for (size_t i = a; i < b; ++i) {
    acc += px[i - a];
    if (cut.size() < (size_t)K && i + 1 < b && acc * K >= total * cut.size()) cut.push_back(i + 1);
  }
  cut.push_back(b);
  const int nk = (int)cut.size() - 1;
  if (upload) maybe_inject(s, PS_INJECT_UPLOAD, "upload states");
  // pinned staging: [uploads (float4)][downloads (float4)][costs (float)]
  float4* stage = (float4*)pinned(s, std::max<size_t>(total, 1) * (2 * sizeof(float4) + sizeof(float)));
  float4* upst = stage;
  float4* dnst = stage + total;
  float* cst = (float*)(stage + 2 * total);
  std::vector<size_t> so(b - a);
  for (size_t i = a, o = 0; i < b; ++i) {
    so[i - a] = o;
    o += px[i - a];
  }
  if (!s->up) cuda_ok(cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking), "cudaStreamCreate");
  if (!s->down) cuda_ok(cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking), "cudaStreamCreate");
  while (s->stage_ev.size() < (size_t)(2 * nk)) {
    cudaEvent_t e;
    cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    s->stage_ev.push_back(e);
  }
  xfer_events(s, b - a);
  auto pack_upload = [&](int k) {
    for (size_t i = cut[k]; i < cut[k + 1]; ++i) {
      const ps_view_state& st = states[i];
      const long long n = (long long)px[i - a];
      float4* q = upst + so[i - a];
#pragma omp parallel for schedule(static) if (n > 65536)
      for (long long q2 = 0; q2 < n; ++q2)
        q[q2] = make_float4(st.normal[3 * q2], st.normal[3 * q2 + 1], st.normal[3 * q2 + 2], st.depth[q2]);
      cuda_ok(cudaMemcpyAsync(sl.plane + sl.off[views[i]], q, (size_t)n * sizeof(float4), cudaMemcpyHostToDevice,
                              s->up),
              "upload planes");
    }
    cuda_ok(cudaEventRecord(s->stage_ev[2 * k], s->up), "cudaEventRecord");
    cuda_ok(cudaStreamWaitEvent(s->st, s->stage_ev[2 * k], 0), "cudaStreamWaitEvent");
  };
  auto download = [&](int k) {
    cuda_ok(cudaStreamWaitEvent(s->down, s->stage_ev[2 * k + 1], 0), "cudaStreamWaitEvent");
    for (size_t i = cut[k]; i < cut[k + 1]; ++i) {
      const size_t n = px[i - a];
      cuda_ok(cudaMemcpyAsync(dnst + so[i - a], sl.plane + sl.off[views[i]], n * sizeof(float4),
                              cudaMemcpyDeviceToHost, s->down),
              "download planes");
      cuda_ok(cudaMemcpyAsync(cst + so[i - a], sl.cost + sl.off[views[i]], n * sizeof(float), cudaMemcpyDeviceToHost,
                              s->down),
              "download cost");
      cuda_ok(cudaEventRecord(s->xfer[i - a], s->down), "cudaEventRecord");
    }
  };
  auto unpack = [&](int k) {
    for (size_t i = cut[k]; i < cut[k + 1]; ++i) {
      cuda_ok(cudaEventSynchronize(s->xfer[i - a]), "cudaEventSynchronize");
      ps_view_state& st = states[i];
      const long long n = (long long)px[i - a];
      const float4* q = dnst + so[i - a];
#pragma omp parallel for schedule(static) if (n > 65536)
      for (long long q2 = 0; q2 < n; ++q2) {
        st.normal[3 * q2] = q[q2].x;
        st.normal[3 * q2 + 1] = q[q2].y;
        st.normal[3 * q2 + 2] = q[q2].z;
        st.depth[q2] = q[q2].w;
      }
      memcpy(st.cost, cst + so[i - a], (size_t)n * sizeof(float));
    }
  };
  for (int k = 0; k < nk; ++k) {
    if (upload) pack_upload(k);
    run_batch(s, views, cut[k], cut[k + 1], p, false);
    cuda_ok(cudaEventRecord(s->stage_ev[2 * k + 1], s->st), "cudaEventRecord");
    download(k);
    if (k > 0) unpack(k - 1);  // chunk k runs meanwhile
  }
  unpack(nk - 1);
  cuda_ok(cudaStreamSynchronize(s->up), "cudaStreamSynchronize");
  sync(s);  // fault and error words
}
}  // namespace

int ps_run(ps_session* s, const uint32_t* views, size_t n, ps_view_state* states, const ps_run_params* p,
           const ps_depth_snapshot* snapshot) {
  return guard(s, [&] {
    if (!p) fail(PS_EINVAL, "params is NULL");
    if (p->random_init > PS_INIT_PROPOSAL) fail(PS_EINVAL, "random_init must be 0, 1 or 2");
    check_views(s, views, n);
    if (n && !states) fail(PS_EINVAL, "states is NULL");
    if (p->geometric) ensure_snapshot(s, snapshot);
    if (p->geometric && s->snap_level != (int)p->level) fail(PS_EINVAL, "snapshot level differs from the run level");
    const int level = (int)p->level;
    Slot& sl = slot(s, level);
    for (auto [a, b] : batches(s, views, n, level)) {
      for (size_t i = a; i < b; ++i) check_state(s, (int)views[i], level, states[i]);
      size_t px = 0;
      for (size_t i = a; i < b; ++i) px += (size_t)states[i].width * states[i].height;
      if (!p->use_prior && p->random_init != PS_INIT_PROPOSAL && b - a >= 2 && px >= kPipelinePixels) {
        run_pipelined(s, views, a, b, states, p);
        continue;
      }
      bool all_prior = true;
      for (size_t i = a; i < b; ++i) all_prior = all_prior && states[i].prior != nullptr;
      if (!p->random_init || (p->use_prior && all_prior)) {
        if (!p->random_init) upload_planes(s, views, a, b, states, level, p->use_prior && all_prior);
        else {
          // prior only: upload it without touching the planes
          for (size_t i = a; i < b; ++i) {
            const size_t np = (size_t)states[i].width * states[i].height;
            cuda_ok(cudaMemcpyAsync(sl.prior + sl.off[views[i]], states[i].prior, np * sizeof(float4),
                                    cudaMemcpyHostToDevice, s->st),
                    "upload prior");
            sl.prior_valid[views[i]] = 1;
          }
          sync(s);
        }
      }
      run_batch(s, views, a, b, p, p->use_prior && all_prior);
      download_states(s, views, a, b, states, level, true, true);
    }
  });
}

int ps_evaluate(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_view_state* states,
                uint32_t geometric, const ps_depth_snapshot* snapshot, float* const* out_cost) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (n && (!states || !out_cost)) fail(PS_EINVAL, "states/out_cost is NULL");
    if (geometric) {
      ensure_snapshot(s, snapshot);
      if (s->snap_level != (int)level) fail(PS_EINVAL, "snapshot level differs from the evaluation level");
    }
    Slot& sl = slot(s, (int)level);
    for (auto [a, b] : batches(s, views, n, (int)level)) {
      upload_planes(s, views, a, b, states, (int)level, false);
      PsRun P = base_params(s, (int)level);
      P.geometric = geometric ? 1 : 0;
      P.mode = 0;
      set_items(s, P, views, a, b, (int)level, PS_EVAL_PW, PS_EVAL_PH);
      timed_launch(s, PS_KERNEL_EVAL, P, [&](const PsRun& q) { return s->L->eval(q, s->tuning & PS_TUNE_TEX_GATHER, s->st); }, "evaluate kernel");
      for (size_t i = a; i < b; ++i) {
        if (!out_cost[i]) fail(PS_EINVAL, "out_cost entry is NULL");
        cuda_ok(cudaMemcpyAsync(out_cost[i], sl.cost + sl.off[views[i]],
                                (size_t)s->W(views[i], level) * s->H(views[i], level) * sizeof(float),
                                cudaMemcpyDeviceToHost, s->st),
                "download cost");
      }
      sync(s);
    }
  });
}

int ps_filter(ps_session* s, const uint32_t* views, size_t n, const ps_view_state* states,
              const ps_depth_snapshot* snapshot, uint8_t* const* out_counts) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (n && (!states || !out_counts)) fail(PS_EINVAL, "states/out_counts is NULL");
    ensure_snapshot(s, snapshot);
    const int level = s->snap_level;
    Slot& sl = slot(s, level);
    for (auto [a, b] : batches(s, views, n, level)) {
      upload_planes(s, views, a, b, states, level, false);
      PsRun P = base_params(s, level);
      P.geometric = 1;
      set_items(s, P, views, a, b, level, PS_EVAL_PW, PS_EVAL_PH);
      timed_launch(s, PS_KERNEL_FILTER, P, [&](const PsRun& q) { return s->L->filter(q, s->tuning & PS_TUNE_TEX_GATHER, s->st); }, "filter kernel");
      for (size_t i = a; i < b; ++i) {
        if (!out_counts[i]) fail(PS_EINVAL, "out_counts entry is NULL");
        cuda_ok(cudaMemcpyAsync(out_counts[i], sl.count + sl.off[views[i]],
                                (size_t)s->W(views[i], level) * s->H(views[i], level), cudaMemcpyDeviceToHost, s->st),
                "download counts");
      }
      sync(s);
    }
  });
}

int ps_upsample(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_view_state* low,
                float sigma_s, float sigma_c, ps_view_state* out) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (level < 1 || level >= (uint32_t)s->nl) fail(PS_EINVAL, "upsample level must be in 1..num_levels-1");
    if (n && (!low || !out)) fail(PS_EINVAL, "low/out is NULL");
    for (auto [a, b] : batches(s, views, n, (int)level)) {
      upload_planes(s, views, a, b, low, (int)level - 1, false);
      PsRun P = base_params(s, (int)level);
      P.prior = s->slots[level - 1].plane;
      P.up_inv2s = 1.0f / (2.0f * sigma_s * sigma_s);
      P.up_inv2c = 1.0f / (2.0f * sigma_c * sigma_c);
      set_items(s, P, views, a, b, (int)level, PS_SIMPLE_BX, PS_SIMPLE_BY, (int)level - 1);
      launched(s, s->L->upsample(P, s->st), "upsample kernel");
      download_states(s, views, a, b, out, (int)level, true, true);
    }
  });
}

int ps_median_filter(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_view_state* in,
                     ps_view_state* out) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (n && (!in || !out)) fail(PS_EINVAL, "in/out is NULL");
    Slot& sl = slot(s, (int)level);
    for (auto [a, b] : batches(s, views, n, (int)level)) {
      upload_planes(s, views, a, b, in, (int)level, false, sl.aux);
      PsRun P = base_params(s, (int)level);
      P.prior = sl.aux;
      set_items(s, P, views, a, b, (int)level, PS_SIMPLE_BX, PS_SIMPLE_BY, (int)level);
      launched(s, s->L->median(P, s->st), "median kernel");
      download_states(s, views, a, b, out, (int)level, true, false);
      for (size_t i = a; i < b; ++i)
        if (out[i].cost && in[i].cost && out[i].cost != in[i].cost)
          memcpy(out[i].cost, in[i].cost, (size_t)in[i].width * in[i].height * sizeof(float));
    }
  });
}

int ps_snapshot_capture(ps_session* s, uint32_t level, const uint32_t* views, size_t n, uint64_t id,
                        uint32_t keep_others) {
  return guard(s, [&] {
    check_views(s, views, n);
    Slot& sl = slot(s, (int)level);
    if ((size_t)sl.total > s->snap_cap) {
      if (keep_others) fail(PS_EINVAL, "keep_others needs a snapshot buffer of this level");
      realloc_snapshot(s, sl.total);
    }
    std::vector<long long> offs(s->nv, -1);
    if (keep_others && s->snap_valid && s->snap_level == (int)level) {
      cuda_ok(cudaMemcpyAsync(offs.data(), s->snap_off, s->nv * sizeof(long long), cudaMemcpyDeviceToHost, s->st), "read offsets");
      sync(s);
      // resident captures always use the slot layout
      for (int v = 0; v < s->nv; ++v)
        if (offs[v] >= 0 && offs[v] != sl.off[v]) fail(PS_EINVAL, "keep_others needs a resident snapshot");
    }
    for (size_t i = 0; i < n; ++i) offs[views[i]] = sl.off[views[i]];
    for (auto [a, b] : batches(s, views, n, (int)level)) {
      PsRun P = base_params(s, (int)level);
      set_items(s, P, views, a, b, (int)level, PS_SIMPLE_BX, PS_SIMPLE_BY, (int)level);
      launched(s, s->L->snapshot(P, s->snap, s->st), "snapshot kernel");
    }
    cuda_ok(cudaMemcpyAsync(s->snap_off, offs.data(), s->nv * sizeof(long long), cudaMemcpyHostToDevice, s->st), "upload offsets");
    sync(s);
    s->snap_valid = true;
    s->snap_level = (int)level;
    s->snap_id = id;
  });
}

int ps_snapshot_buffer(ps_session* s, uint32_t level, float** device_ptr, uint64_t* offsets) {
  return guard(s, [&] {
    Slot& sl = slot(s, (int)level);
    if ((size_t)sl.total > s->snap_cap || s->snap_level != (int)level) {
      // (re)lay the buffer out like the level's slots; nothing is present yet
      if ((size_t)sl.total > s->snap_cap) {
        realloc_snapshot(s, sl.total);
      }
      std::vector<long long> none(s->nv, -1);
      cuda_ok(cudaMemcpyAsync(s->snap_off, none.data(), s->nv * sizeof(long long), cudaMemcpyHostToDevice, s->st),
              "upload offsets");
      sync(s);
      s->snap_level = (int)level;
      s->snap_valid = false;
    }
    if (device_ptr) *device_ptr = s->snap;
    if (offsets)
      for (int v = 0; v < s->nv; ++v) offsets[v] = (uint64_t)sl.off[v];
  });
}

int ps_snapshot_mark(ps_session* s, uint32_t level, const uint32_t* views, size_t n, uint64_t id) {
  return guard(s, [&] {
    check_views(s, views, n);
    Slot& sl = slot(s, (int)level);
    if (s->snap_level != (int)level || (size_t)sl.total > s->snap_cap)
      fail(PS_EINVAL, "call ps_snapshot_buffer for this level first");
    std::vector<long long> offs(s->nv, -1);
    cuda_ok(cudaMemcpyAsync(offs.data(), s->snap_off, s->nv * sizeof(long long), cudaMemcpyDeviceToHost, s->st),
            "read offsets");
    sync(s);
    for (size_t i = 0; i < n; ++i) offs[views[i]] = sl.off[views[i]];
    cuda_ok(cudaMemcpyAsync(s->snap_off, offs.data(), s->nv * sizeof(long long), cudaMemcpyHostToDevice, s->st),
            "upload offsets");
    sync(s);
    s->snap_valid = true;
    s->snap_id = id;
  });
}

int ps_filter_resident(ps_session* s, const uint32_t* views, size_t n, uint8_t* const* out_counts) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (!s->snap_valid) fail(PS_EINVAL, "filter needs a snapshot");
    const int level = s->snap_level;
    Slot& sl = slot(s, level);
    for (auto [a, b] : batches(s, views, n, level)) {
      PsRun P = base_params(s, level);
      P.geometric = 1;
      set_items(s, P, views, a, b, level, PS_EVAL_PW, PS_EVAL_PH);
      timed_launch(s, PS_KERNEL_FILTER, P, [&](const PsRun& q) { return s->L->filter(q, s->tuning & PS_TUNE_TEX_GATHER, s->st); }, "filter kernel");
      if (out_counts) {
        for (size_t i = a; i < b; ++i)
          if (out_counts[i])
            cuda_ok(cudaMemcpyAsync(out_counts[i], sl.count + sl.off[views[i]],
                                    (size_t)s->W(views[i], level) * s->H(views[i], level), cudaMemcpyDeviceToHost, s->st),
                    "download counts");
      }
    }
    if (out_counts) sync(s);
  });
}

int ps_readout_resident(ps_session* s, const uint32_t* views, size_t n, ps_view_state* out) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (!s->snap_valid) fail(PS_EINVAL, "readout needs the filter's snapshot level");
    const int level = s->snap_level;
    Slot& sl = slot(s, level);
    for (auto [a, b] : batches(s, views, n, level)) {
      PsRun P = base_params(s, level);
      set_items(s, P, views, a, b, level, PS_SIMPLE_BX, PS_SIMPLE_BY);
      launched(s, s->L->readout(P, sl.aux, s->st), "readout kernel");
      if (out) download_states(s, views, a, b, out, level, true, true, sl.aux);
    }
  });
}

namespace {

// Snapshot of `views` at `level` captured on the device: depth of the resident planes into the snapshot buffer (slot
// layout) and the offset table copied from a device array prepared for this view set.  No host synchronisation.
void enqueue_snapshot(ps_session* s, const uint32_t* views, size_t n, int level, const long long* offsets_dev) {
  for (auto [a, b] : batches(s, views, n, level)) {
    PsRun P = base_params(s, level);
    set_items(s, P, views, a, b, level, PS_SIMPLE_BX, PS_SIMPLE_BY, level);
    launched(s, s->L->snapshot(P, s->snap, s->st), "snapshot kernel");
  }
  cuda_ok(cudaMemcpyAsync(s->snap_off, offsets_dev, s->nv * sizeof(long long), cudaMemcpyDeviceToDevice, s->st),
          "snapshot offsets");
}

// The launches of one single-level schedule, in the order of densify.schedule_resident.
void enqueue_schedule(ps_session* s, const uint32_t* views, size_t n, const ps_schedule* sch,
                      const long long* offsets_dev) {
  const int level = (int)sch->level;
  Slot& sl = slot(s, level);
  ps_run_params p{sch->level, 0, sch->init == PS_INIT_PROPOSAL ? PS_INIT_PROPOSAL : PS_INIT_RANDOM,
                  sch->photometric_iters, sch->run_id_base, 0};
  for (auto [a, b] : batches(s, views, n, level)) run_batch(s, views, a, b, &p, false);
  for (uint32_t r = 0; r < sch->geometric_rounds; ++r) {
    enqueue_snapshot(s, views, n, level, offsets_dev);
    ps_run_params g{sch->level, 1, 0, sch->geometric_iters, sch->run_id_base + 1 + r, 0};
    for (auto [a, b] : batches(s, views, n, level)) run_batch(s, views, a, b, &g, false);
  }
  enqueue_snapshot(s, views, n, level, offsets_dev);
  for (auto [a, b] : batches(s, views, n, level)) {
    PsRun P = base_params(s, level);
    P.geometric = 1;
    set_items(s, P, views, a, b, level, PS_EVAL_PW, PS_EVAL_PH);
    timed_launch(s, PS_KERNEL_FILTER, P, [&](const PsRun& q) { return s->L->filter(q, s->tuning & PS_TUNE_TEX_GATHER, s->st); }, "filter kernel");
    PsRun Q = base_params(s, level);
    set_items(s, Q, views, a, b, level, PS_SIMPLE_BX, PS_SIMPLE_BY);
    launched(s, s->L->readout(Q, sl.aux, s->st), "readout kernel");
  }
}

}  // namespace

extern "C++" {
namespace {

// The launches of the multi-scale driver (densify.compute_depth_maps with the restorer's default: no random init):
// coarsest level from random init; every finer level upsampled (joint bilateral), evaluated, refined by a restorer
// run from the upsampled planes, evaluated again and merged per pixel (k_restore); geometric rounds at every level
// against snapshots captured on the device; at the top level the median filter (when the filter parameters ask for
// it), the final snapshot, the filter and the readout.  Run ids count up from run_id_base like the host driver's.
void enqueue_multiscale(ps_session* s, const uint32_t* views, size_t n, const ps_multiscale_schedule* m,
                        const std::vector<long long*>& offs) {
  uint32_t run_id = m->run_id_base;
  const int top = s->nl - 1;
  for (int l = 0; l < s->nl; ++l) {
    Slot& sl = slot(s, l);
    const uint32_t iters = l == 0 ? m->photometric_iters : m->photometric_iters_upper;
    const bool use_prior = l > 0 && m->weak_texture_prior && s->pm.weak_texture_var > 0.0f;
    if (l == 0) {
      ps_run_params p{0, 0, PS_INIT_RANDOM, iters, run_id++, 0};
      for (auto [a, b] : batches(s, views, n, 0)) run_batch(s, views, a, b, &p, false);
    } else {
      for (auto [a, b] : batches(s, views, n, l)) {
        PsRun U = base_params(s, l);
        U.prior = s->slots[l - 1].plane;
        U.up_inv2s = 1.0f / (2.0f * m->jbu_sigma_spatial * m->jbu_sigma_spatial);
        U.up_inv2c = 1.0f / (2.0f * m->jbu_sigma_color * m->jbu_sigma_color);
        set_items(s, U, views, a, b, l, PS_SIMPLE_BX, PS_SIMPLE_BY, l - 1);
        launched(s, s->L->upsample(U, s->st), "upsample kernel");
        PsRun E = base_params(s, l);  // c_init: top-K photometric cost of the upsampled planes
        set_items(s, E, views, a, b, l, PS_EVAL_PW, PS_EVAL_PH);
        timed_launch(s, PS_KERNEL_EVAL, E, [&](const PsRun& q) { return s->L->eval(q, s->tuning & PS_TUNE_TEX_GATHER, s->st); }, "evaluate kernel");
      }
      for (size_t i = 0; i < n; ++i) {  // keep the upsampled planes and their cost
        const size_t np = (size_t)s->W(views[i], l) * s->H(views[i], l), o = (size_t)sl.off[views[i]];
        cuda_ok(cudaMemcpyAsync(sl.aux + o, sl.plane + o, np * sizeof(float4), cudaMemcpyDeviceToDevice, s->st), "copy");
        cuda_ok(cudaMemcpyAsync(sl.cinit + o, sl.cost + o, np * sizeof(float), cudaMemcpyDeviceToDevice, s->st), "copy");
        if (use_prior)
          cuda_ok(cudaMemcpyAsync(sl.prior + o, sl.plane + o, np * sizeof(float4), cudaMemcpyDeviceToDevice, s->st),
                  "copy");
      }
      ps_run_params p{(uint32_t)l, 0, 0, iters, run_id++, use_prior ? 1u : 0u};
      for (auto [a, b] : batches(s, views, n, l)) run_batch(s, views, a, b, &p, use_prior);
      for (auto [a, b] : batches(s, views, n, l)) {
        PsRun E = base_params(s, l);  // c_photo
        set_items(s, E, views, a, b, l, PS_EVAL_PW, PS_EVAL_PH);
        timed_launch(s, PS_KERNEL_EVAL, E, [&](const PsRun& q) { return s->L->eval(q, s->tuning & PS_TUNE_TEX_GATHER, s->st); }, "evaluate kernel");
        PsRun R = base_params(s, l);
        set_items(s, R, views, a, b, l, PS_SIMPLE_BX, PS_SIMPLE_BY);
        launched(s, s->L->restore(R, sl.aux, sl.cinit, m->restorer_threshold, s->st), "restore kernel");
      }
    }
    for (uint32_t r = 0; r < m->geometric_rounds; ++r) {
      enqueue_snapshot(s, views, n, l, offs[l]);
      ps_run_params g{(uint32_t)l, 1, 0, m->geometric_iters, run_id++, use_prior ? 1u : 0u};
      for (auto [a, b] : batches(s, views, n, l)) run_batch(s, views, a, b, &g, use_prior);
    }
  }
  Slot& st = slot(s, top);
  if (s->fl.median_filter) {
    for (size_t i = 0; i < n; ++i) {
      const size_t np = (size_t)s->W(views[i], top) * s->H(views[i], top), o = (size_t)st.off[views[i]];
      cuda_ok(cudaMemcpyAsync(st.aux + o, st.plane + o, np * sizeof(float4), cudaMemcpyDeviceToDevice, s->st), "copy");
    }
    for (auto [a, b] : batches(s, views, n, top)) {
      PsRun M = base_params(s, top);
      M.prior = st.aux;
      set_items(s, M, views, a, b, top, PS_SIMPLE_BX, PS_SIMPLE_BY, top);
      launched(s, s->L->median(M, s->st), "median kernel");
    }
  }
  enqueue_snapshot(s, views, n, top, offs[top]);
  for (auto [a, b] : batches(s, views, n, top)) {
    PsRun P = base_params(s, top);
    P.geometric = 1;
    set_items(s, P, views, a, b, top, PS_EVAL_PW, PS_EVAL_PH);
    timed_launch(s, PS_KERNEL_FILTER, P, [&](const PsRun& q) { return s->L->filter(q, s->tuning & PS_TUNE_TEX_GATHER, s->st); }, "filter kernel");
    PsRun Q = base_params(s, top);
    set_items(s, Q, views, a, b, top, PS_SIMPLE_BX, PS_SIMPLE_BY);
    launched(s, s->L->readout(Q, st.aux, s->st), "readout kernel");
  }
}

// Runs `enqueue` through a CUDA graph captured once per key (use_graph) or directly; `prepare` allocates and uploads
// what the launches need, outside any capture.
template <typename Prep, typename Enq>
void graph_run(ps_session* s, const std::string& key, bool use_graph, Prep&& prepare, Enq&& enqueue) {
  auto it = s->graphs.find(key);
  if (it == s->graphs.end()) {
    ps_session::GraphEntry ge;
    auto release = [&] {
      dfree(s, ge.offsets);
      for (long long* o : ge.level_offsets) dfree(s, o);
    };
    try {
      prepare(ge);
      sync(s);
    } catch (...) {
      release();
      throw;
    }
    if (use_graph) {
      // capture once: the launches the direct path issues, recorded into a graph; with profiling on, the per-launch
      // events become event-record nodes that every replay re-records
      collect_events(s);
      const uint64_t before = s->launches;
      uint64_t kl[PS_KERNEL_KINDS];
      for (int k = 0; k < PS_KERNEL_KINDS; ++k) kl[k] = s->kind_launches[k];
      cudaGraph_t g = nullptr;
      cuda_ok(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
      s->capturing = true;
      try {
        enqueue(ge);
        s->capturing = false;
      } catch (...) {
        s->capturing = false;
        cudaStreamEndCapture(s->st, &g);
        if (g) cudaGraphDestroy(g);
        s->launches = before;
        for (auto& pd : s->pending) {
          cudaEventDestroy(pd.a);
          cudaEventDestroy(pd.b);
        }
        s->pending.clear();
        release();
        throw;
      }
      ge.per_replay = s->launches - before;
      s->launches = before;
      for (int k = 0; k < PS_KERNEL_KINDS; ++k) s->kind_launches[k] = kl[k];
      ge.events = s->pending;
      for (auto& pd : ge.events) pd.persistent = true;
      s->pending.clear();
      cudaError_t e = cudaStreamEndCapture(s->st, &g);
      if (e == cudaSuccess) e = cudaGraphInstantiate(&ge.exec, g, 0);
      if (g) cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        release();
        for (auto& pd : ge.events) {
          cudaEventDestroy(pd.a);
          cudaEventDestroy(pd.b);
        }
      }
      cuda_ok(e, "graph capture");
    }
    it = s->graphs.emplace(key, ge).first;
  }
  ps_session::GraphEntry& ge = it->second;
  if (ge.exec) {
    if (!ge.events.empty()) collect_events(s);  // the previous replay's event nodes are re-recorded by this one
    cuda_ok(cudaGraphLaunch(ge.exec, s->st), "cudaGraphLaunch");
    s->launches += ge.per_replay;
    for (auto& pd : ge.events) {
      s->pending.push_back(pd);
      s->kind_launches[pd.kind]++;
    }
  } else {
    enqueue(ge);
  }
}

void ensure_snapshot_capacity(ps_session* s, long long total) {
  if ((size_t)total > s->snap_cap) {
    realloc_snapshot(s, total);  // drops captured graphs: they hold the old buffer's address
  }
}

long long* view_offsets(ps_session* s, int level, const uint32_t* views, size_t n) {
  Slot& sl = slot(s, level);
  std::vector<long long> offs(s->nv, -1);
  for (size_t i = 0; i < n; ++i) offs[views[i]] = sl.off[views[i]];
  long long* d = dalloc<long long>(s, s->nv);
  cuda_ok(cudaMemcpyAsync(d, offs.data(), s->nv * sizeof(long long), cudaMemcpyHostToDevice, s->st), "upload offsets");
  return d;
}

}  // namespace
}  // extern "C++"

int ps_schedule_resident(ps_session* s, const uint32_t* views, size_t n, const ps_schedule* sch) {
  return guard(s, [&] {
    if (!sch) fail(PS_EINVAL, "schedule is NULL");
    if (sch->init > PS_INIT_PROPOSAL) fail(PS_EINVAL, "schedule init must be PS_INIT_RANDOM or PS_INIT_PROPOSAL");
    check_views(s, views, n);
    const int level = (int)sch->level;
    Slot& sl = slot(s, level);
    ensure_snapshot_capacity(s, sl.total);  // the snapshot buffer in the slot layout, allocated outside any capture
    std::string key = "single:" + std::to_string(level) + ":" + std::to_string(sch->photometric_iters) + ":" +
                      std::to_string(sch->geometric_rounds) + ":" + std::to_string(sch->geometric_iters) + ":" +
                      std::to_string(sch->run_id_base) + ":" + std::to_string(sch->use_graph) + ":" +
                      std::to_string(s->profiling) + ":" + std::to_string(sch->init == PS_INIT_PROPOSAL) + ":";
    for (size_t i = 0; i < n; ++i) key += std::to_string(views[i]) + ",";
    graph_run(
        s, key, sch->use_graph != 0,
        [&](ps_session::GraphEntry& ge) { ge.offsets = view_offsets(s, level, views, n); },
        [&](ps_session::GraphEntry& ge) { enqueue_schedule(s, views, n, sch, ge.offsets); });
    s->snap_valid = true;
    s->snap_level = level;
    s->snap_id = 0x5c4ed000ull + sch->run_id_base;
  });
}

void ps_multiscale_schedule_default(ps_multiscale_schedule* out) {
  if (!out) return;
  memset(out, 0, sizeof *out);
  out->photometric_iters = 6;
  out->photometric_iters_upper = 3;
  out->geometric_rounds = 2;
  out->geometric_iters = 2;
  out->jbu_sigma_spatial = 1.0f;
  out->jbu_sigma_color = 0.04f;
  out->restorer_threshold = 0.1f;
  out->weak_texture_prior = 0;
  out->run_id_base = 1;
  out->use_graph = 1;
}

int ps_schedule_multiscale(ps_session* s, const uint32_t* views, size_t n, const ps_multiscale_schedule* m) {
  return guard(s, [&] {
    if (!m) fail(PS_EINVAL, "schedule is NULL");
    if (!(m->jbu_sigma_spatial > 0.f) || !(m->jbu_sigma_color > 0.f)) fail(PS_EINVAL, "JBU sigmas must be > 0");
    check_views(s, views, n);
    const int top = s->nl - 1;
    for (int l = 0; l < s->nl; ++l) {  // every buffer the launches use exists before any capture
      Slot& sl = slot(s, l);
      if (l > 0 && !sl.cinit) sl.cinit = dalloc<float>(s, std::max<long long>(sl.total, 1));
    }
    long long maxtot = 0;
    for (int l = 0; l < s->nl; ++l) maxtot = std::max(maxtot, s->slots[l].total);
    ensure_snapshot_capacity(s, maxtot);
    char buf[256];
    snprintf(buf, sizeof buf, "multi:%u:%u:%u:%u:%a:%a:%a:%u:%u:%u:%d:", m->photometric_iters,
             m->photometric_iters_upper, m->geometric_rounds, m->geometric_iters, m->jbu_sigma_spatial,
             m->jbu_sigma_color, m->restorer_threshold, m->weak_texture_prior, m->run_id_base, m->use_graph,
             (int)s->profiling);
    std::string key = buf;
    for (size_t i = 0; i < n; ++i) key += std::to_string(views[i]) + ",";
    graph_run(
        s, key, m->use_graph != 0,
        [&](ps_session::GraphEntry& ge) {
          for (int l = 0; l < s->nl; ++l) ge.level_offsets.push_back(view_offsets(s, l, views, n));
        },
        [&](ps_session::GraphEntry& ge) { enqueue_multiscale(s, views, n, m, ge.level_offsets); });
    s->snap_valid = true;
    s->snap_level = top;
    s->snap_id = 0x3c4ed000ull + m->run_id_base;
  });
}


// ---- learned proposal ------------------------------------------------------------------------------------------
extern "C++" {
namespace {

void ensure_proposals(ps_session* s, Slot& sl) {
  if (sl.proposal) return;
  sl.proposal = dalloc<float4>(s, sl.total);
  sl.pconf = dalloc<float>(s, sl.total);
  cuda_ok(cudaMemsetAsync(sl.proposal, 0, std::max<long long>(sl.total, 1) * sizeof(float4), s->st), "memset");
  cuda_ok(cudaMemsetAsync(sl.pconf, 0, std::max<long long>(sl.total, 1) * sizeof(float), s->st), "memset");
  sl.proposal_valid.assign(s->nv, 0);
}

void enqueue_sweep(ps_session* s, int level, uint32_t view, unsigned short* out, int row_pixels) {
  PsRun P = base_params(s, level);
  P.netin = out;
  P.netin_pitch = row_pixels;
  P.sweep_ws = 2;
  for (int c = 0; c < 3; ++c) P.sweep_n[c] = s->sweep_n[3 * view + c];
  set_items(s, P, &view, 0, 1, level, PS_EVAL_PW, PS_EVAL_PH);
  const bool tex = (s->tuning & PS_TUNE_TEX_GATHER) != 0;  // the session built texture objects for its planes
  timed_launch(s, PS_KERNEL_SWEEP, P, [&](const PsRun& q) { return s->L->sweep(q, tex, s->st); }, "sweep kernel");
}

template <typename T>
void grow(ps_session* s, T*& buf, size_t& cap, size_t elems) {
  if (elems <= cap) return;
  sync(s);  // the previous user of the buffer has finished
  dfree(s, buf);
  buf = nullptr;
  cap = 0;
  buf = dalloc<T>(s, elems);
  cap = elems;
}

}  // namespace
}  // extern "C++"

int ps_set_sweep_normals(ps_session* s, const float* normals) {
  return guard(s, [&] {
    for (int v = 0; v < s->nv; ++v) {
      const float* n = normals ? normals + 3 * v : nullptr;
      const float x = n ? n[0] : 0.0f, y = n ? n[1] : 0.0f, z = n ? n[2] : -1.0f;
      const float len = std::sqrt(x * x + y * y + z * z);
      if (!(len > 0.5f && len < 2.0f) || !(z < 0.0f)) fail(PS_EINVAL, "sweep normal of view " + std::to_string(v) +
                                                               " must be a unit vector facing the camera (z < 0)");
      s->sweep_n[3 * v] = x;
      s->sweep_n[3 * v + 1] = y;
      s->sweep_n[3 * v + 2] = z;
    }
  });
}

int ps_sweep_volume(ps_session* s, uint32_t level, uint32_t view, void* out, uint32_t row_pixels) {
  return guard(s, [&] {
    check_views(s, &view, 1);
    if (!out) fail(PS_EINVAL, "out is NULL");
    slot(s, (int)level);
    if ((int)row_pixels < s->W((int)view, (int)level)) fail(PS_EINVAL, "row_pixels is smaller than the view width");
    if ((uintptr_t)out % 16) fail(PS_EINVAL, "out must be 16-byte aligned");
    enqueue_sweep(s, (int)level, view, (unsigned short*)out, (int)row_pixels);
  });
}

int ps_propose(ps_session* s, ps_net* net, uint32_t level, const uint32_t* views, size_t n, float conf_threshold,
               uint64_t* proposed) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (!net) fail(PS_EINVAL, "net is NULL");
    if (!(conf_threshold >= 0.f && conf_threshold <= 1.f)) fail(PS_EINVAL, "conf_threshold must be in [0, 1]");
    const int l = (int)level;
    Slot& sl = slot(s, l);
    ensure_proposals(s, sl);
    size_t in_need = 1, out_need = 1;
    for (size_t i = 0; i < n; ++i) {
      const size_t hp = round_up(s->H(views[i], l), 8), wp = round_up(s->W(views[i], l), 8);
      in_need = std::max(in_need, hp * wp * PS_NET_CH_IN);
      out_need = std::max(out_need, hp * wp * PS_NET_CH_OUT);
    }
    grow(s, s->netin, s->netin_cap, in_need);
    grow(s, s->netout, s->netout_cap, out_need);
    if (!s->pcount) s->pcount = dalloc<unsigned long long>(s, 2);  // two counters (post-processing uses both)
    cuda_ok(cudaMemsetAsync(s->pcount, 0, sizeof(unsigned long long), s->st), "memset");
    for (size_t i = 0; i < n; ++i) {
      const uint32_t v = views[i];
      const int w = s->W(v, l), h = s->H(v, l);
      const int hp = (int)round_up(h, 8), wp = (int)round_up(w, 8);
      if (hp != h || wp != w)
        cuda_ok(cudaMemsetAsync(s->netin, 0, (size_t)hp * wp * PS_NET_CH_IN * 2, s->st), "memset");
      enqueue_sweep(s, l, v, s->netin, wp);
      ps_session::Pending pd{};
      if (s->profiling) {
        cuda_ok(cudaEventCreate(&pd.a), "cudaEventCreate");
        cuda_ok(cudaEventCreate(&pd.b), "cudaEventCreate");
        cuda_ok(cudaEventRecord(pd.a, s->st), "cudaEventRecord");
      }
      std::string err;
      const int rc = ps_cnn::forward_on_stream(net, s->netin, 1, hp, wp, s->netout, s->st, &err);
      if (rc != PS_OK) {
        if (s->profiling) {
          cudaEventDestroy(pd.a);
          cudaEventDestroy(pd.b);
        }
        fail(rc, "proposal network: " + err);
      }
      const PsLevel& L = s->lvh[v * s->nl + l];
      const float k[4] = {L.fx, L.fy, L.cx, L.cy};
      const PsView& vd = s->vdh[v];
      cuda_ok(ps_cnn::launch_decode(s->netout, wp, h, w, sl.proposal + sl.off[v], sl.pconf + sl.off[v],
                                    1.0f / vd.dmin, 1.0f / vd.dmax, conf_threshold, k, s->pcount, s->st),
              "decode kernel");
      s->launches += ps_cnn::kForwardLaunches + 1;
      if (s->profiling) {
        cuda_ok(cudaEventRecord(pd.b, s->st), "cudaEventRecord");
        pd.kind = PS_KERNEL_NET;
        pd.persistent = false;
        s->pending.push_back(pd);
        s->kind_launches[PS_KERNEL_NET]++;
      }
      sl.proposal_valid[v] = 1;
    }
    if (proposed) {
      unsigned long long c = 0;
      cuda_ok(cudaMemcpyAsync(&c, s->pcount, sizeof c, cudaMemcpyDeviceToHost, s->st), "read proposal count");
      sync(s);
      *proposed = c;
      std::string e;
      const int h = ps_cnn::conv_health(&e);
      if (h != PS_OK) fail(h, "proposal network: " + e);
    }
  });
}

int ps_proposal_upload(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const float* const* planes) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (n && !planes) fail(PS_EINVAL, "planes is NULL");
    Slot& sl = slot(s, (int)level);
    ensure_proposals(s, sl);
    for (size_t i = 0; i < n; ++i) {
      if (!planes[i]) fail(PS_EINVAL, "planes[i] is NULL");
      const size_t np = (size_t)s->W(views[i], (int)level) * s->H(views[i], (int)level);
      cuda_ok(cudaMemcpyAsync(sl.proposal + sl.off[views[i]], planes[i], np * sizeof(float4), cudaMemcpyHostToDevice,
                              s->st),
              "upload proposal");
    }
    sync(s);
    for (size_t i = 0; i < n; ++i) sl.proposal_valid[views[i]] = 1;
  });
}

int ps_proposal_download(ps_session* s, uint32_t level, const uint32_t* views, size_t n, float* const* planes,
                         float* const* conf) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (n && !planes) fail(PS_EINVAL, "planes is NULL");
    Slot& sl = slot(s, (int)level);
    for (size_t i = 0; i < n; ++i)
      if (!sl.proposal || !sl.proposal_valid[views[i]])
        fail(PS_EINVAL, "view " + std::to_string(views[i]) + " has no proposal");
    for (size_t i = 0; i < n; ++i) {
      const size_t np = (size_t)s->W(views[i], (int)level) * s->H(views[i], (int)level);
      if (!planes[i]) fail(PS_EINVAL, "planes[i] is NULL");
      cuda_ok(cudaMemcpyAsync(planes[i], sl.proposal + sl.off[views[i]], np * sizeof(float4), cudaMemcpyDeviceToHost,
                              s->st),
              "download proposal");
      if (conf && conf[i])
        cuda_ok(cudaMemcpyAsync(conf[i], sl.pconf + sl.off[views[i]], np * sizeof(float), cudaMemcpyDeviceToHost,
                                s->st),
                "download confidence");
    }
    sync(s);
  });
}

int ps_readout_download(ps_session* s, uint32_t level, const uint32_t* views, size_t n, ps_view_state* out) {
  return guard(s, [&] {
    check_views(s, views, n);
    if (n && !out) fail(PS_EINVAL, "out is NULL");
    Slot& sl = slot(s, (int)level);
    for (auto [a, b] : batches(s, views, n, (int)level)) download_states(s, views, a, b, out, (int)level, true, true, sl.aux);
  });
}

// ---- post-processing and fusion --------------------------------------------------------------------------------
extern "C++" {
namespace {

// Item table of a speckle / count launch over views[a..b) at `level` (32 × 8 pixel tiles).
int spk_items(ps_session* s, ps_post::SpkArgs& A, const uint32_t* views, size_t a, size_t b, int level, double frac) {
  Slot& sl = s->slots[level];
  int tiles = 0;
  A.nitems = (int)(b - a);
  for (size_t i = a; i < b; ++i) {
    const int v = (int)views[i];
    ps_post::SpkItem& it = A.items[i - a];
    it.off = sl.off[v];
    it.w = s->W(v, level);
    it.h = s->H(v, level);
    it.tile0 = tiles;
    it.min_area = (int)std::ceil((double)it.w * it.h * frac);
    tiles += ((it.w + 31) / 32) * ((it.h + 7) / 8);
  }
  return tiles;
}

}  // namespace
}  // extern "C++"

void ps_post_params_default(ps_post_params* out) {
  if (!out) return;
  out->remove_speckles = 1;
  out->speckle_rel_depth = 0.02f;
  out->speckle_min_area_frac = 2e-4;
  out->speckle_keep_cost = 0.2f;
  out->fill_holes = 0;
  out->fill_max_frac = 0.01;
  out->fill_edge_step = 0.06f;
  out->fill_max_cost = 1.0f;
}

void ps_fusion_params_default(ps_fusion_params* out) {
  if (!out) return;
  memset(out, 0, sizeof *out);
  out->min_consistent_views = 5;
  out->consistency_num_images = 12;
  out->mark_used = 1;
  out->mark_radius = 0;
  out->inverse_variance = 1;
  out->sigma_px0 = 0.25;
  out->sigma_px_slope = 1.0;
  out->max_reproj_error = 2.0;
  out->max_depth_error = 0.01;
  out->max_normal_error_deg = 10.0;
  out->residual = PS_FUSION_RESIDUAL_NONE;
  out->residual_min_views = 2;
  out->residual_depth_error = std::numeric_limits<double>::quiet_NaN();
  out->residual_normal_error_deg = std::numeric_limits<double>::quiet_NaN();
  out->residual_min_dist_gsd = 0.5;
  out->visibility_check_views = 0;
  out->visibility_min_violations = 2;
  out->visibility_tau = 0.01;
  out->smooth_iterations = 0;
  out->smooth_radius_gsd = 1.0;
  out->smooth_sigma_range_gsd = 0.25;
  out->smooth_normal_deg = 30.0;
}

int ps_postprocess_resident(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_post_params* p,
                            const double* intrinsics, uint64_t* removed, uint64_t* filled) {
  return guard(s, [&] {
    if (!p) fail(PS_EINVAL, "params is NULL");
    check_views(s, views, n);
    if (level >= (uint32_t)s->nl) fail(PS_EINVAL, "level out of range");
    Slot& sl = slot(s, (int)level);
    if (removed) *removed = 0;
    if (filled) *filled = 0;
    if (n == 0 || (!p->remove_speckles && !p->fill_holes)) return;
    if (!sl.spk) sl.spk = dalloc<int>(s, (size_t)std::max<long long>(sl.total, 1) * 5);
    if (!s->pcount) s->pcount = dalloc<unsigned long long>(s, 2);
    cuda_ok(cudaMemsetAsync(s->pcount, 0, 2 * sizeof(unsigned long long), s->st), "memset");
    const size_t T = (size_t)std::max<long long>(sl.total, 1);
    if (p->remove_speckles)
    for (auto [a, b] : batches(s, views, n, (int)level)) {
      ps_post::SpkArgs A;
      memset(&A, 0, sizeof A);
      A.plane = sl.aux;
      A.cost = sl.cost;
      A.parent = sl.spk;
      A.size = sl.spk + T;
      A.lo = (unsigned*)(sl.spk + 2 * T);
      A.hi = (unsigned*)(sl.spk + 3 * T);
      A.cnt = (unsigned*)(sl.spk + 4 * T);
      A.removed = s->pcount;
      A.rel = p->speckle_rel_depth;
      A.keep = p->speckle_keep_cost;
      const int tiles = spk_items(s, A, views, a, b, (int)level, p->speckle_min_area_frac);
      bool any = false;
      for (int i = 0; i < A.nitems; ++i) any = any || A.items[i].min_area > 1;
      if (!any) continue;  // the reference returns early when the minimum area is <= 1
      for (int i = 0; i < A.nitems; ++i)
        if (A.items[i].min_area <= 1) A.items[i].min_area = 0;  // no component is small
      int nl = 0;
      cuda_ok(ps_post::launch_speckles(A, tiles, s->st, &nl), "speckle kernels");
      s->launches += nl;
    }
    if (p->fill_holes) {
      // scratch: a float4 fill plane and a cost per slot pixel in the speckle buffer (5 words per pixel)
      float4* tplane = reinterpret_cast<float4*>(sl.spk);
      float* tcost = reinterpret_cast<float*>(sl.spk + 4 * T);
      for (size_t i = 0; i < n; ++i) {
        const int v = (int)views[i];
        const PsLevel& L = s->lvh[v * s->nl + (int)level];
        ps_post::FillArgs F;
        memset(&F, 0, sizeof F);
        F.plane = sl.aux + sl.off[v];
        F.cost = sl.cost + sl.off[v];
        F.img = L.img;
        F.pitch = L.pitch;
        F.tplane = tplane + sl.off[v];
        F.tcost = tcost + sl.off[v];
        F.filled = s->pcount + 1;
        F.w = s->W(v, (int)level);
        F.h = s->H(v, (int)level);
        if (intrinsics) {
          for (int k = 0; k < 4; ++k) F.k[k] = intrinsics[4 * v + k];
        } else {
          F.k[0] = L.fx;
          F.k[1] = L.fy;
          F.k[2] = L.cx;
          F.k[3] = L.cy;
        }
        const long long W = F.w, H = F.h;
        F.maxd = (int)std::max<long long>((long long)std::round(std::sqrt((double)(W * W + H * H)) * p->fill_max_frac), 1);
        F.step = (int)(p->fill_edge_step * 255.0f);
        F.max_cost = p->fill_max_cost;
        launched(s, ps_post::launch_fill_holes(F, s->st), "hole filling kernels");
        s->launches += 1;  // two kernels per view (launched() counts one)
      }
    }
    if (removed || filled) {
      unsigned long long c[2] = {0, 0};
      cuda_ok(cudaMemcpyAsync(c, s->pcount, sizeof c, cudaMemcpyDeviceToHost, s->st), "read counts");
      sync(s);
      if (removed) *removed = c[0];
      if (filled) *filled = c[1];
    }
  });
}

namespace {
// Valid pixels (depth > 0) of the readout planes of `views` at level l.
unsigned long long count_valid(ps_session* s, const uint32_t* views, size_t n, int l) {
  Slot& sl = slot(s, l);
  FusedCloud& fc = s->fused;
  if (!fc.counter) fc.counter = dalloc<unsigned long long>(s, 1);
  cuda_ok(cudaMemsetAsync(fc.counter, 0, sizeof(unsigned long long), s->st), "memset");
  for (auto [a, b] : batches(s, views, n, l)) {
    ps_post::SpkArgs A;
    memset(&A, 0, sizeof A);
    A.plane = sl.aux;
    A.valid = fc.counter;
    const int tiles = spk_items(s, A, views, a, b, l, 0.0);
    cuda_ok(ps_post::launch_count_valid(A, tiles, s->st), "count kernel");
    s->launches++;
  }
  unsigned long long valid = 0;
  cuda_ok(cudaMemcpyAsync(&valid, fc.counter, sizeof valid, cudaMemcpyDeviceToHost, s->st), "read count");
  sync(s);
  return valid;
}

// Ground sample distance (depth_gsd, crates/dense/src/fusion.rs:469-487) of the fused views `order` (ascending).
double fused_gsd(ps_session* s, Slot& sl, const std::vector<uint32_t>& order, const ps_fusion_view* cams, int l) {
  std::vector<ps_post::GsdView> gv(order.size());
  long long soff = 0;
  for (size_t i = 0; i < order.size(); ++i) {
    const int v = (int)order[i];
    gv[i].off = sl.off[v];
    gv[i].npix = s->W(v, l) * s->H(v, l);
    gv[i].soff = soff;
    gv[i].fx = cams[v].k[0];
    soff += (gv[i].npix + 96) / 97;
  }
  ps_post::GsdView* dgv = dalloc<ps_post::GsdView>(s, gv.size());
  float* samples = dalloc<float>(s, std::max<long long>(soff, 1));
  unsigned* scount = dalloc<unsigned>(s, gv.size());
  double* dgsd = dalloc<double>(s, gv.size());
  cuda_ok(cudaMemcpyAsync(dgv, gv.data(), gv.size() * sizeof(ps_post::GsdView), cudaMemcpyHostToDevice, s->st),
          "upload gsd views");
  launched(s, ps_post::launch_gsd(sl.aux, dgv, (int)gv.size(), samples, scount, dgsd, s->st), "gsd kernel");
  std::vector<double> gs(gv.size());
  cuda_ok(cudaMemcpyAsync(gs.data(), dgsd, gs.size() * sizeof(double), cudaMemcpyDeviceToHost, s->st), "read gsd");
  sync(s);
  dfree(s, dgv);
  dfree(s, samples);
  dfree(s, scount);
  dfree(s, dgsd);
  std::vector<double> g2;
  for (double x : gs)
    if (!std::isnan(x)) g2.push_back(x);
  double gsd = 0.0;
  if (!g2.empty()) {  // median_in_place (crates/dense/src/math.rs:137-141)
    std::sort(g2.begin(), g2.end());
    const double pos = 0.5 * (double)(g2.size() - 1);
    const size_t lo = (size_t)std::floor(pos), hi = std::min(lo + 1, g2.size() - 1);
    gsd = g2[lo] + (g2[hi] - g2[lo]) * (pos - (double)lo);
  }
  return gsd;
}

// filter_visibility (crates/dense/src/visibility.rs:106-151) of the fused cloud, when p turns it on.  masked: only the
// points whose keep entry is set are tested (the others stay out and are not counted); otherwise every point is, and
// the keep mask is made here.
void fused_visibility(ps_session* s, Slot& sl, FusedCloud& fc, const ps_fusion_view* cams,
                      const std::vector<char>& used, const ps_fusion_params* p, bool masked) {
  const bool vis_on = p->visibility_check_views > 0 && p->visibility_tau > 0.0 && p->visibility_min_violations > 0;
  if (!vis_on || fc.count == 0) return;
  if (p->visibility_check_views > PS_VIS_MAX_CHECK) fail(PS_EINVAL, "visibility_check_views > 64");
  // full overlap lists of the fused views (the candidate order of the filter)
  std::vector<int> ovoff(s->nv + 1, 0), ovlist;
  for (int v = 0; v < s->nv; ++v) {
    ovoff[v] = (int)ovlist.size();
    if (!used[v]) continue;
    for (uint32_t j = 0; j < cams[v].num_overlap; ++j) ovlist.push_back((int)cams[v].overlap[j]);
  }
  ovoff[s->nv] = (int)ovlist.size();
  std::vector<unsigned char> used8(used.begin(), used.end());
  int* dovoff = dalloc<int>(s, ovoff.size());
  int* dovlist = dalloc<int>(s, std::max<size_t>(ovlist.size(), 1));
  unsigned char* dused = dalloc<unsigned char>(s, std::max(s->nv, 1));
  unsigned long long* drem = dalloc<unsigned long long>(s, 2);
  if (!masked) fc.keep = dalloc<unsigned char>(s, fc.count);
  cuda_ok(cudaMemcpyAsync(dovoff, ovoff.data(), ovoff.size() * sizeof(int), cudaMemcpyHostToDevice, s->st), "upload");
  if (!ovlist.empty())
    cuda_ok(cudaMemcpyAsync(dovlist, ovlist.data(), ovlist.size() * sizeof(int), cudaMemcpyHostToDevice, s->st),
            "upload");
  cuda_ok(cudaMemcpyAsync(dused, used8.data(), used8.size(), cudaMemcpyHostToDevice, s->st), "upload");
  cuda_ok(cudaMemsetAsync(drem, 0, 2 * sizeof(unsigned long long), s->st), "memset");
  ps_post::VisArgs V;
  memset(&V, 0, sizeof V);
  V.views = fc.views;
  V.plane = sl.aux;
  V.used = dused;
  V.ovoff = dovoff;
  V.ovlist = dovlist;
  V.nviews = s->nv;
  V.pos = fc.pos;
  V.nvis = fc.nvis;
  V.vis = fc.vis;
  V.vis_stride = fc.vis_stride;
  V.n = fc.count;
  V.n1 = fc.count1;
  V.limit = (int)p->visibility_check_views;
  V.min_violations = (int)p->visibility_min_violations;
  V.tau = p->visibility_tau;
  V.keep = fc.keep;
  V.masked = masked ? 1 : 0;
  V.removed = drem;
  launched(s, ps_post::launch_visibility(V, s->st), "visibility kernel");
  unsigned long long rem[2] = {0, 0};
  cuda_ok(cudaMemcpyAsync(rem, drem, sizeof rem, cudaMemcpyDeviceToHost, s->st), "read counts");
  sync(s);
  fc.removed1 = rem[0];
  fc.removed2 = rem[1];
  dfree(s, dovoff);
  dfree(s, dovlist);
  dfree(s, dused);
  dfree(s, drem);
}

// smooth_along_normals (crates/dense/src/smooth.rs:143-220) of the kept points, as densify.rs:552-556 runs it, when p
// turns it on; the neighbour order is the cloud order (candidate numbers after score fusion).
void fused_smoothing(ps_session* s, Slot& sl, FusedCloud& fc, const std::vector<uint32_t>& order,
                     const ps_fusion_view* cams, int l, const ps_fusion_params* p) {
  const bool smooth_on = p->smooth_iterations > 0 && p->smooth_radius_gsd > 0.0 && p->smooth_sigma_range_gsd > 0.0;
  if (!smooth_on || fc.count == 0) return;
  const double gsd = fused_gsd(s, sl, order, cams, l);
  if (gsd > 0.0) {
    ps_post::SmoothArgs M;
    memset(&M, 0, sizeof M);
    M.r = p->smooth_radius_gsd * gsd;
    M.r2 = M.r * M.r;
    M.inv_2ss = 1.0 / (2.0 * ((0.5 * M.r) * (0.5 * M.r)));
    const double sr = p->smooth_sigma_range_gsd * gsd;
    M.inv_2sr = 1.0 / (2.0 * (sr * sr));
    M.cos_n = std::cos(ps_to_radians_f64(p->smooth_normal_deg));
    M.n = fc.count;
    M.n1 = fc.count1;
    M.nrm = fc.nrm;
    M.keep = fc.keep;
    M.key = fc.key;
    M.gid = fc.gid;
    unsigned cap = 1024;
    while (cap < 2ull * fc.count) cap <<= 1;
    M.cap = cap;
    M.hkeys = dalloc<unsigned long long>(s, cap);
    M.hcnt = dalloc<unsigned>(s, cap);
    M.hstart = dalloc<unsigned>(s, cap);
    M.hcur = dalloc<unsigned>(s, cap);
    M.list = dalloc<unsigned>(s, fc.count);
    M.pslot = dalloc<unsigned>(s, fc.count);
    M.total = dalloc<unsigned>(s, 1);
    M.flag = dalloc<int>(s, 1);
    float* pos2 = dalloc<float>(s, 3 * fc.count);
    cuda_ok(cudaMemcpyAsync(pos2, fc.pos, 12 * fc.count, cudaMemcpyDeviceToDevice, s->st), "copy");
    cuda_ok(cudaMemsetAsync(M.flag, 0, sizeof(int), s->st), "memset");
    float* cur = fc.pos;
    float* nxt = pos2;
    for (uint32_t it = 0; it < p->smooth_iterations; ++it) {
      cuda_ok(cudaMemsetAsync(M.hkeys, 0, cap * sizeof(unsigned long long), s->st), "memset");
      cuda_ok(cudaMemsetAsync(M.hcnt, 0, cap * sizeof(unsigned), s->st), "memset");
      cuda_ok(cudaMemsetAsync(M.hcur, 0, cap * sizeof(unsigned), s->st), "memset");
      cuda_ok(cudaMemsetAsync(M.total, 0, sizeof(unsigned), s->st), "memset");
      M.pos = cur;
      M.pos2 = nxt;
      cuda_ok(ps_post::launch_smooth_pass(M, s->st), "smoothing kernels");
      s->launches += 5;
      std::swap(cur, nxt);
    }
    if (cur != fc.pos)
      cuda_ok(cudaMemcpyAsync(fc.pos, cur, 12 * fc.count, cudaMemcpyDeviceToDevice, s->st), "copy");
    int flag = 0;
    cuda_ok(cudaMemcpyAsync(&flag, M.flag, sizeof flag, cudaMemcpyDeviceToHost, s->st), "read flag");
    sync(s);
    for (void* q : {(void*)M.hkeys, (void*)M.hcnt, (void*)M.hstart, (void*)M.hcur, (void*)M.list, (void*)M.pslot,
                    (void*)M.total, (void*)M.flag, (void*)pos2})
      dfree(s, q);
    if (flag) fail(PS_EINVAL, "smoothing: a point lies more than 2^20 smoothing radii from the origin");
  }
}
}  // namespace

int ps_fuse_resident(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_fusion_view* cams,
                     const ps_fusion_params* p, uint64_t* num_points, uint64_t* num_residual) {
  return guard(s, [&] {
    if (!p || (n && !cams)) fail(PS_EINVAL, "params or cams is NULL");
    if (p->residual > PS_FUSION_RESIDUAL_SECOND_PASS) fail(PS_EINVAL, "residual must be 0, 1 or 2");
    const bool second = p->residual == PS_FUSION_RESIDUAL_SECOND_PASS;
    check_views(s, views, n);
    if (s->nv > 65535) fail(PS_EINVAL, "fusion supports at most 65535 views");
    if (p->consistency_num_images > PS_FUSE_MAX_OVERLAP)
      fail(PS_EINVAL, "consistency_num_images > " + std::to_string(PS_FUSE_MAX_OVERLAP));
    const int l = (int)level;
    Slot& sl = slot(s, l);
    std::vector<char> used(s->nv, 0);
    for (size_t i = 0; i < n; ++i) used[views[i]] = 1;
    // camera table (indexed by session view); overlap lists filtered to used views and truncated
    std::vector<ps_post::FuseView> fv(s->nv);
    for (int v = 0; v < s->nv; ++v) {
      ps_post::FuseView& f = fv[v];
      memset(&f, 0, sizeof f);
      f.off = sl.off[v];
      f.w = s->W(v, l);
      f.h = s->H(v, l);
      const PsLevel& L = s->lvh[v * s->nl + l];
      f.img = L.img;
      f.pitch = L.pitch;
      if (!used[v]) continue;
      const ps_fusion_view& c = cams[v];
      memcpy(f.k, c.k, sizeof f.k);
      memcpy(f.r, c.r, sizeof f.r);
      memcpy(f.t, c.t, sizeof f.t);
      f.baseline = c.baseline;
      f.image_id = c.image_id;
      if (c.num_overlap && !c.overlap) fail(PS_EINVAL, "overlap is NULL");
      for (uint32_t j = 0; j < c.num_overlap && f.nov < (int)p->consistency_num_images; ++j) {
        const uint32_t o = c.overlap[j];
        if (o >= (uint32_t)s->nv) fail(PS_EINVAL, "overlap view out of range");
        if (used[o] && (int)o != v) f.ov[f.nov++] = (int)o;
      }
    }
    FusedCloud& fc = s->fused;
    if (!fc.counter) fc.counter = dalloc<unsigned long long>(s, 1);
    if (!fc.views) fc.views = dalloc<ps_post::FuseView>(s, std::max(s->nv, 1));
    cuda_ok(cudaMemcpyAsync(fc.views, fv.data(), fv.size() * sizeof(ps_post::FuseView), cudaMemcpyHostToDevice, s->st),
            "upload fusion views");
    const unsigned long long valid = count_valid(s, views, n, l);  // capacity
    const int stride = (int)p->consistency_num_images + 1;
    if (valid > fc.cap || stride != fc.vis_stride) {
      fc.release([s](void* q) { dfree(s, q); });
      const size_t c = std::max<unsigned long long>(valid, 1);
      fc.pos = dalloc<float>(s, 3 * c);
      fc.nrm = dalloc<float>(s, 3 * c);
      fc.col = dalloc<unsigned char>(s, 3 * c);
      fc.key = dalloc<unsigned long long>(s, c);
      fc.nvis = dalloc<unsigned char>(s, c);
      fc.vis = dalloc<unsigned short>(s, c * stride);
      fc.cap = c;
      fc.vis_stride = stride;
    }
    {  // key order = the fused views in ascending image id, row-major within a view
      std::vector<std::pair<unsigned, int>> iv;
      for (int v = 0; v < s->nv; ++v)
        if (used[v]) iv.push_back({cams[v].image_id, v});
      std::sort(iv.begin(), iv.end());
      fc.ids.clear();
      fc.bases.clear();
      fc.widths.clear();
      fc.cells = 0;
      fc.ordered = true;
      for (size_t i = 0; i < iv.size(); ++i) {
        if (i && iv[i].first == iv[i - 1].first) fc.ordered = false;
        fc.ids.push_back(iv[i].first);
        fc.bases.push_back(fc.cells);
        fc.widths.push_back(s->W(iv[i].second, l));
        fc.cells += (unsigned long long)s->W(iv[i].second, l) * s->H(iv[i].second, l);
      }
    }
    if (!sl.marks) sl.marks = dalloc<unsigned char>(s, std::max<long long>(sl.total, 1));
    cuda_ok(cudaMemsetAsync(sl.marks, 0, std::max<long long>(sl.total, 1), s->st), "memset");
    cuda_ok(cudaMemsetAsync(fc.counter, 0, sizeof(unsigned long long), s->st), "memset");
    ps_post::FuseArgs A;
    memset(&A, 0, sizeof A);
    A.views = fc.views;
    A.plane = sl.aux;
    A.cost = sl.cost;
    A.marks = sl.marks;
    A.min_views = (int)p->min_consistent_views;
    A.mark_used = p->mark_used ? 1 : 0;
    A.mark_radius = (int)p->mark_radius;
    A.inverse_variance = p->inverse_variance ? 1 : 0;
    A.sigma0 = p->sigma_px0;
    A.slope = p->sigma_px_slope;
    A.depth_tol = p->max_depth_error;
    A.cos_n = std::cos(ps_to_radians_f64(p->max_normal_error_deg));
    A.r2 = p->max_reproj_error * p->max_reproj_error;
    A.pos = fc.pos;
    A.nrm = fc.nrm;
    A.col = fc.col;
    A.key = fc.key;
    A.nvis = fc.nvis;
    A.vis = fc.vis;
    A.vis_stride = stride;
    A.count = fc.counter;
    A.capacity = fc.cap;
    std::vector<uint32_t> order(views, views + n);
    std::sort(order.begin(), order.end());  // the reference walks views in index order
    order.erase(std::unique(order.begin(), order.end()), order.end());
    if (second) {
      if (!sl.consumed) sl.consumed = dalloc<unsigned char>(s, std::max<long long>(sl.total, 1));
      cuda_ok(cudaMemsetAsync(sl.consumed, 0, std::max<long long>(sl.total, 1), s->st), "memset");
      A.consumed = sl.consumed;
    }
    for (uint32_t v : order) {
      A.v = (int)v;
      cuda_ok(ps_post::launch_fuse(A, s->W(v, l), s->H(v, l), s->st), "fusion kernel");
      s->launches++;
    }
    unsigned long long cnt = 0;
    cuda_ok(cudaMemcpyAsync(&cnt, fc.counter, sizeof cnt, cudaMemcpyDeviceToHost, s->st), "read count");
    sync(s);
    fc.count1 = std::min(cnt, fc.cap);
    if (second) {
      const double gsd = fused_gsd(s, sl, order, cams, l);
      const double min_dist = p->residual_min_dist_gsd * gsd;
      // candidate numbers: prefix of the fused views' pixel counts in index order (fusion.rs:560-565)
      std::vector<ps_post::FuseView> fv2 = fv;
      unsigned long long base = 0;
      for (int v = 0; v < s->nv; ++v) {
        fv2[v].idbase = (unsigned)base;
        if (used[v]) base += (unsigned long long)s->W(v, l) * s->H(v, l);
      }
      if (base >= 0xffffffffull) fail(PS_EINVAL, "second pass: more than 2^32 - 1 pixels");
      cuda_ok(cudaMemcpyAsync(fc.views, fv2.data(), fv2.size() * sizeof(ps_post::FuseView), cudaMemcpyHostToDevice,
                              s->st),
              "upload fusion views");
      unsigned* owner = dalloc<unsigned>(s, std::max<long long>(sl.total, 1));
      cuda_ok(cudaMemsetAsync(owner, 0xff, std::max<long long>(sl.total, 1) * sizeof(unsigned), s->st), "memset");
      unsigned long long* gkeys = nullptr;
      unsigned *gheads = nullptr, *gnext = nullptr;
      int* overflow = nullptr;
      unsigned cap = 0;
      const unsigned n1 = (unsigned)fc.count1;
      if (min_dist > 0.0 && n1 > 0) {
        cap = 1024;
        while (cap < 2u * n1) cap <<= 1;
        gkeys = dalloc<unsigned long long>(s, cap);
        gheads = dalloc<unsigned>(s, cap);
        gnext = dalloc<unsigned>(s, n1);
        overflow = dalloc<int>(s, 1);
        cuda_ok(cudaMemsetAsync(gkeys, 0, cap * sizeof(unsigned long long), s->st), "memset");
        cuda_ok(cudaMemsetAsync(gheads, 0xff, cap * sizeof(unsigned), s->st), "memset");
        cuda_ok(cudaMemsetAsync(overflow, 0, sizeof(int), s->st), "memset");
        launched(s, ps_post::launch_grid_insert(fc.pos, n1, min_dist, gkeys, gheads, gnext, cap, overflow, s->st),
                 "grid kernel");
      }
      ps_post::FuseArgs B = A;
      B.depth_tol = std::isnan(p->residual_depth_error) ? 0.5 * p->max_depth_error : p->residual_depth_error;
      B.cos_n = std::cos(ps_to_radians_f64(std::isnan(p->residual_normal_error_deg) ? 0.67 * p->max_normal_error_deg
                                                                                    : p->residual_normal_error_deg));
      B.min_views = (int)p->residual_min_views;
      B.owner = owner;
      B.gkeys = gkeys;
      B.gheads = gheads;
      B.gnext = gnext;
      B.gcap = cap;
      B.gpoints = n1;
      B.gcell = min_dist;
      for (int stage = 1; stage <= 2; ++stage)
        for (uint32_t v : order) {
          B.v = (int)v;
          cuda_ok(ps_post::launch_fuse_second(B, s->W(v, l), s->H(v, l), stage, s->st), "second-pass kernel");
          s->launches++;
        }
      int ovf = 0;
      cuda_ok(cudaMemcpyAsync(&cnt, fc.counter, sizeof cnt, cudaMemcpyDeviceToHost, s->st), "read count");
      if (overflow) cuda_ok(cudaMemcpyAsync(&ovf, overflow, sizeof ovf, cudaMemcpyDeviceToHost, s->st), "read flag");
      sync(s);
      dfree(s, owner);
      dfree(s, gkeys);
      dfree(s, gheads);
      dfree(s, gnext);
      dfree(s, overflow);
      if (ovf) fail(PS_ECUDA, "second pass: spatial hash table full");
    }
    fc.count = std::min(cnt, fc.cap);
    fc.removed1 = fc.removed2 = fc.rejected = 0;
    if (fc.keep) dfree(s, fc.keep);
    fc.keep = nullptr;
    if (fc.gid) dfree(s, fc.gid);
    fc.gid = nullptr;
    fused_visibility(s, sl, fc, cams, used, p, false);
    fused_smoothing(s, sl, fc, order, cams, l, p);
    if (num_points) *num_points = fc.count - fc.removed1 - fc.removed2;
    if (num_residual) *num_residual = fc.count - fc.count1 - fc.removed2;
  });
}

int ps_fused_visibility_removed(ps_session* s, uint64_t* removed) {
  return guard(s, [&] {
    if (!removed) fail(PS_EINVAL, "removed is NULL");
    *removed = s->fused.removed1 + s->fused.removed2;
  });
}

void ps_score_fusion_params_default(ps_score_fusion_params* out) {
  if (!out) return;
  memset(out, 0, sizeof *out);
  out->sigma_e_px = 1.0;
  out->sigma_theta_deg = 2.0;
  out->lambda = 1.0;
  out->tau = 2.0;
  out->depth_error = 0.01;
  out->normal_error_deg = 10.0;
  out->num_neighbors = 12;
  out->mark_used = 1;
  out->inverse_variance = 1;
  out->sigma_px0 = 0.25;
  out->sigma_px_slope = 1.0;
}

// fuse_scored (crates/dense/src/fusion_score.rs:314-435): candidates per view (one launch per fused view, in index
// order), then with mark_used the adoption rounds until no candidate is undecided (the host reads the undecided count
// every few rounds; a round adopts at least the highest-priority undecided candidate, so rounds <= candidates); then
// the visibility filter and the smoothing of `post` on the adopted points.
int ps_fuse_scored_resident(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_fusion_view* cams,
                            const ps_score_fusion_params* p, const ps_fusion_params* post, uint64_t* num_points) {
  return guard(s, [&] {
    if (!p || (n && !cams)) fail(PS_EINVAL, "params or cams is NULL");
    check_views(s, views, n);
    if (s->nv > 65535) fail(PS_EINVAL, "fusion supports at most 65535 views");
    if (p->num_neighbors > PS_FUSE_MAX_OVERLAP) fail(PS_EINVAL, "num_neighbors > " + std::to_string(PS_FUSE_MAX_OVERLAP));
    const int l = (int)level;
    Slot& sl = slot(s, l);
    if (sl.total >= 0xffffffffLL) fail(PS_EINVAL, "score fusion: more than 2^32 - 1 pixels in the level");
    std::vector<char> used(s->nv, 0);
    for (size_t i = 0; i < n; ++i) used[views[i]] = 1;
    // camera table: overlap lists without the view itself and unused or out-of-range views, first num_neighbors
    // (fusion_score.rs:324-330); candidate numbers in (view, pixel) order over the fused views
    std::vector<ps_post::FuseView> fv(s->nv);
    unsigned long long base = 0;
    for (int v = 0; v < s->nv; ++v) {
      ps_post::FuseView& f = fv[v];
      memset(&f, 0, sizeof f);
      f.off = sl.off[v];
      f.w = s->W(v, l);
      f.h = s->H(v, l);
      const PsLevel& L = s->lvh[v * s->nl + l];
      f.img = L.img;
      f.pitch = L.pitch;
      f.idbase = (unsigned)base;
      if (!used[v]) continue;
      base += (unsigned long long)f.w * f.h;
      const ps_fusion_view& c = cams[v];
      memcpy(f.k, c.k, sizeof f.k);
      memcpy(f.r, c.r, sizeof f.r);
      memcpy(f.t, c.t, sizeof f.t);
      f.baseline = c.baseline;
      f.image_id = c.image_id;
      if (c.num_overlap && !c.overlap) fail(PS_EINVAL, "overlap is NULL");
      for (uint32_t j = 0; j < c.num_overlap && f.nov < (int)p->num_neighbors; ++j) {
        const uint32_t o = c.overlap[j];
        if (o < (uint32_t)s->nv && (int)o != v && used[o]) f.ov[f.nov++] = (int)o;
      }
    }
    if (base >= 0xfffffffeull) fail(PS_EINVAL, "score fusion: more than 2^32 - 2 pixels");
    FusedCloud& fc = s->fused;
    if (!fc.views) fc.views = dalloc<ps_post::FuseView>(s, std::max(s->nv, 1));
    cuda_ok(cudaMemcpyAsync(fc.views, fv.data(), fv.size() * sizeof(ps_post::FuseView), cudaMemcpyHostToDevice, s->st),
            "upload fusion views");
    const unsigned long long valid = count_valid(s, views, n, l);  // capacity
    const int stride = (int)p->num_neighbors + 1;
    const unsigned long long score_cells = base;  // candidate numbers run over the fused views' pixels
    if (valid > fc.cap || stride != fc.vis_stride) {
      fc.release([s](void* q) { dfree(s, q); });
      const size_t c = std::max<unsigned long long>(valid, 1);
      fc.pos = dalloc<float>(s, 3 * c);
      fc.nrm = dalloc<float>(s, 3 * c);
      fc.col = dalloc<unsigned char>(s, 3 * c);
      fc.key = dalloc<unsigned long long>(s, c);
      fc.nvis = dalloc<unsigned char>(s, c);
      fc.vis = dalloc<unsigned short>(s, c * stride);
      fc.cap = c;
      fc.vis_stride = stride;
    }
    if (fc.keep) dfree(s, fc.keep);
    if (fc.gid) dfree(s, fc.gid);
    fc.keep = dalloc<unsigned char>(s, fc.cap);
    fc.gid = dalloc<unsigned>(s, fc.cap);
    fc.count = fc.count1 = fc.removed1 = fc.removed2 = fc.rejected = 0;
    fc.ids.clear();
    fc.bases.clear();
    fc.widths.clear();
    fc.cells = score_cells;
    fc.ordered = true;
    ps_post::ScoreArgs A;
    memset(&A, 0, sizeof A);
    A.views = fc.views;
    A.plane = sl.aux;
    A.cost = sl.cost;
    A.inverse_variance = p->inverse_variance ? 1 : 0;
    A.mark_used = p->mark_used ? 1 : 0;
    A.sigma0 = p->sigma_px0;
    A.slope = p->sigma_px_slope;
    A.depth_tol = p->depth_error;
    A.cos_n = std::cos(ps_to_radians_f64(p->normal_error_deg));
    A.k_e = 1.0 / (2.0 * p->sigma_e_px * p->sigma_e_px);
    const double st = ps_to_radians_f64(p->sigma_theta_deg);
    A.k_t = 1.0 / (2.0 * st * st);
    A.lambda = p->lambda;
    A.tau = p->tau;
    A.pos = fc.pos;
    A.nrm = fc.nrm;
    A.col = fc.col;
    A.key = fc.key;
    A.nvis = fc.nvis;
    A.vis = fc.vis;
    A.vis_stride = stride;
    A.gid = fc.gid;
    A.state = fc.keep;
    A.count = fc.counter;
    A.capacity = fc.cap;
    A.prio = dalloc<unsigned long long>(s, fc.cap);
    A.pix = dalloc<unsigned>(s, fc.cap * stride);
    A.npix = dalloc<unsigned char>(s, fc.cap);
    A.pix_stride = stride;
    std::vector<uint32_t> order(views, views + n);
    std::sort(order.begin(), order.end());
    order.erase(std::unique(order.begin(), order.end()), order.end());
    cuda_ok(cudaMemsetAsync(fc.counter, 0, sizeof(unsigned long long), s->st), "memset");
    for (uint32_t v : order) {
      A.v = (int)v;
      launched(s, ps_post::launch_score_candidates(A, s->W(v, l), s->H(v, l), s->st), "score fusion kernel");
    }
    unsigned long long cand = 0;
    cuda_ok(cudaMemcpyAsync(&cand, fc.counter, sizeof cand, cudaMemcpyDeviceToHost, s->st), "read count");
    sync(s);
    cand = std::min(cand, fc.cap);
    unsigned long long adopted = cand;
    if (p->mark_used && cand > 0) {
      A.claim = dalloc<unsigned long long>(s, sl.total);
      unsigned* lists = dalloc<unsigned>(s, 2 * cand);
      unsigned* counts = dalloc<unsigned>(s, 2);
      A.adopted = dalloc<unsigned long long>(s, 1);
      cuda_ok(cudaMemsetAsync(A.claim, 0xff, sl.total * sizeof(unsigned long long), s->st), "memset");
      cuda_ok(cudaMemsetAsync(A.adopted, 0, sizeof(unsigned long long), s->st), "memset");
      A.active = lists;
      A.ncur = counts;
      launched(s, ps_post::launch_score_init(A, (unsigned)cand, s->st), "score fusion kernel");
      const int blocks = (int)std::min<unsigned long long>((cand + 255) / 256, 148ull * 16);
      unsigned left = 1;
      for (unsigned long long r = 0; left > 0; ++r) {
        if (r > cand + 8) fail(PS_ECUDA, "score fusion: adoption rounds did not finish");
        A.active = lists + (r & 1) * cand;
        A.next = lists + ((r + 1) & 1) * cand;
        A.ncur = counts + (r & 1);
        A.nnext = counts + ((r + 1) & 1);
        cuda_ok(ps_post::launch_score_round(A, blocks, s->st), "score fusion rounds");
        s->launches += 3;
        if (r % 4 == 3 || r < 4) {
          cuda_ok(cudaMemcpyAsync(&left, A.nnext, sizeof left, cudaMemcpyDeviceToHost, s->st), "read count");
          sync(s);
        }
      }
      cuda_ok(cudaMemcpyAsync(&adopted, A.adopted, sizeof adopted, cudaMemcpyDeviceToHost, s->st), "read count");
      sync(s);
      dfree(s, A.claim);
      dfree(s, lists);
      dfree(s, counts);
      dfree(s, A.adopted);
    }
    dfree(s, A.prio);
    dfree(s, A.pix);
    dfree(s, A.npix);
    fc.count = fc.count1 = cand;
    fc.rejected = cand - adopted;
    if (post) {  // fuse_depth_maps_with (crates/dense/src/densify.rs:535-556): on the adopted points
      fused_visibility(s, sl, fc, cams, used, post, true);
      fused_smoothing(s, sl, fc, order, cams, l, post);
    }
    if (num_points) *num_points = adopted - fc.removed1;
  });
}

namespace {
// The fused cloud in output order, ordered on the device (CloudOrderArgs in csrc/ps_post.h): every kept point marks
// its cell of the output-order grid, an exclusive prefix sum of the marks gives each point's output index, the points
// are scattered into output buffers, and those are copied into the caller's arrays.  Returns false (nothing written)
// when the marks do not count exactly `kept` points, so the caller falls back to ordering on the host.
bool fused_points_device(ps_session* s, size_t kept, float* positions, float* normals, uint8_t* colors, uint64_t* keys,
                         uint8_t* vis_counts, uint16_t* vis, uint32_t vis_stride) {
  FusedCloud& fc = s->fused;
  const size_t n = fc.count;
  const size_t ncell = (fc.gid ? 1 : 2) * (size_t)fc.cells;
  if (ncell >= 0xffffffffull) return false;  // 32-bit ranks
  std::vector<void*> tmp;
  auto get = [&](size_t bytes) {
    void* p = dalloc<unsigned char>(s, std::max<size_t>(bytes, 1));
    tmp.push_back(p);
    return p;
  };
  ps_post::CloudOrderArgs A;
  memset(&A, 0, sizeof A);
  A.n = n;
  A.count1 = std::min<size_t>(fc.count1, n);
  A.cells = fc.cells;
  A.keep = fc.keep;
  A.gid = fc.gid;
  A.key = fc.key;
  A.pos = fc.pos;
  A.nrm = fc.nrm;
  A.col = fc.col;
  A.nvis = fc.nvis;
  A.vis = fc.vis;
  A.vis_stride = fc.vis_stride;
  A.rank = (unsigned*)get((ncell + 1) * sizeof(unsigned));
  unsigned* scratch = (unsigned*)get(ps_post::scan_scratch(ncell + 1) * sizeof(unsigned));
  if (!fc.gid) {
    A.nids = (int)fc.ids.size();
    unsigned* ids = (unsigned*)get(fc.ids.size() * sizeof(unsigned));
    unsigned long long* base = (unsigned long long*)get(fc.bases.size() * sizeof(unsigned long long));
    int* width = (int*)get(fc.widths.size() * sizeof(int));
    cuda_ok(cudaMemcpyAsync(ids, fc.ids.data(), fc.ids.size() * sizeof(unsigned), cudaMemcpyHostToDevice, s->st),
            "upload cloud order");
    cuda_ok(cudaMemcpyAsync(base, fc.bases.data(), fc.bases.size() * sizeof(unsigned long long),
                            cudaMemcpyHostToDevice, s->st),
            "upload cloud order");
    cuda_ok(cudaMemcpyAsync(width, fc.widths.data(), fc.widths.size() * sizeof(int), cudaMemcpyHostToDevice, s->st),
            "upload cloud order");
    A.ids = ids;
    A.base = base;
    A.width = width;
  }
  if (positions) A.opos = (float*)get(kept * 12);
  if (normals) A.onrm = (float*)get(kept * 12);
  if (colors) A.ocol = (unsigned char*)get(kept * 3);
  if (keys) A.okey = (unsigned long long*)get(kept * 8);
  if (vis_counts) A.onvis = (unsigned char*)get(kept);
  if (vis) {
    A.ovis = (unsigned short*)get(kept * vis_stride * sizeof(unsigned short));
    A.ovis_stride = (int)vis_stride;
  }
  cuda_ok(cudaMemsetAsync(A.rank, 0, (ncell + 1) * sizeof(unsigned), s->st), "memset");
  launched(s, ps_post::launch_cloud_mark(A, s->st), "cloud order kernel");
  launched(s, ps_post::scan_exclusive(A.rank, ncell + 1, scratch, s->st), "scan kernel");
  unsigned occupied = 0;
  cuda_ok(cudaMemcpyAsync(&occupied, A.rank + ncell, sizeof occupied, cudaMemcpyDeviceToHost, s->st), "read count");
  sync(s);
  bool ok = occupied == kept;
  if (ok) {
    launched(s, ps_post::launch_cloud_scatter(A, s->st), "cloud scatter kernel");
    auto down = [&](void* dst, const void* src, size_t bytes) {
      if (dst && bytes) cuda_ok(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->st), "download cloud");
    };
    down(positions, A.opos, kept * 12);
    down(normals, A.onrm, kept * 12);
    down(colors, A.ocol, kept * 3);
    down(keys, A.okey, kept * 8);
    down(vis_counts, A.onvis, kept);
    down(vis, A.ovis, kept * vis_stride * sizeof(unsigned short));
    sync(s);
  }
  for (void* p : tmp) dfree(s, p);
  return ok;
}
}  // namespace

int ps_fused_points(ps_session* s, uint64_t capacity, float* positions, float* normals, uint8_t* colors,
                    uint64_t* keys, uint8_t* vis_counts, uint16_t* vis, uint32_t vis_stride) {
  return guard(s, [&] {
    FusedCloud& fc = s->fused;
    const size_t n = fc.count;  // emitted points (before the visibility filter)
    const size_t kept = n - fc.removed1 - fc.removed2 - fc.rejected;
    if (capacity < kept)
      fail(PS_EINVAL, "capacity " + std::to_string(capacity) + " < " + std::to_string(kept) + " points");
    if (vis && (int)vis_stride < fc.vis_stride) fail(PS_EINVAL, "vis_stride too small");
    if (fc.ordered && n && fused_points_device(s, kept, positions, normals, colors, keys, vis_counts, vis, vis_stride))
      return;
    std::vector<float> p(3 * n), q(3 * n);
    std::vector<unsigned char> c(3 * n), nv(n);
    std::vector<unsigned long long> k(n);
    std::vector<unsigned short> vv((size_t)n * std::max(fc.vis_stride, 1));
    if (n) {
      cuda_ok(cudaMemcpyAsync(p.data(), fc.pos, 12 * n, cudaMemcpyDeviceToHost, s->st), "download");
      cuda_ok(cudaMemcpyAsync(q.data(), fc.nrm, 12 * n, cudaMemcpyDeviceToHost, s->st), "download");
      cuda_ok(cudaMemcpyAsync(c.data(), fc.col, 3 * n, cudaMemcpyDeviceToHost, s->st), "download");
      cuda_ok(cudaMemcpyAsync(k.data(), fc.key, 8 * n, cudaMemcpyDeviceToHost, s->st), "download");
      cuda_ok(cudaMemcpyAsync(nv.data(), fc.nvis, n, cudaMemcpyDeviceToHost, s->st), "download");
      cuda_ok(cudaMemcpyAsync(vv.data(), fc.vis, 2 * n * fc.vis_stride, cudaMemcpyDeviceToHost, s->st), "download");
    }
    std::vector<unsigned char> keep(n, 1);
    if (n && fc.keep) cuda_ok(cudaMemcpyAsync(keep.data(), fc.keep, n, cudaMemcpyDeviceToHost, s->st), "download");
    std::vector<unsigned> gid(fc.gid ? n : 0);
    if (n && fc.gid) cuda_ok(cudaMemcpyAsync(gid.data(), fc.gid, 4 * n, cudaMemcpyDeviceToHost, s->st), "download");
    sync(s);
    // points in the reference's order: the first pass, then the second, each in ascending key (view, row, column),
    // without the points the visibility filter removed
    const size_t n1 = std::min<size_t>(fc.count1, n);
    std::vector<size_t> idx;
    idx.reserve(kept);
    for (size_t i = 0; i < n1; ++i)
      if (keep[i]) idx.push_back(i);
    const size_t k1 = idx.size();
    for (size_t i = n1; i < n; ++i)
      if (keep[i]) idx.push_back(i);
    if (fc.gid) {  // score fusion: (view, pixel) order
      std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return gid[a] < gid[b]; });
    } else {
      std::sort(idx.begin(), idx.begin() + k1, [&](size_t a, size_t b) { return k[a] < k[b]; });
      std::sort(idx.begin() + k1, idx.end(), [&](size_t a, size_t b) { return k[a] < k[b]; });
    }
    for (size_t j = 0; j < idx.size(); ++j) {
      const size_t i = idx[j];
      if (positions) memcpy(positions + 3 * j, &p[3 * i], 12);
      if (normals) memcpy(normals + 3 * j, &q[3 * i], 12);
      if (colors) memcpy(colors + 3 * j, &c[3 * i], 3);
      if (keys) keys[j] = k[i];
      if (vis_counts) vis_counts[j] = nv[i];
      if (vis)
        for (int t = 0; t < (int)vis_stride; ++t)
          vis[(size_t)j * vis_stride + t] = t < fc.vis_stride && t < nv[i] ? vv[i * fc.vis_stride + t] : 0;
    }
  });
}

// build_pyramid (crates/dense/src/upsample.rs:46-102) on the GPU.  Weights g = (e^-2, 1, e^-2) / ((e^-2 + 1) + e^-2)
// in binary32 (f32::exp of -1/(2·0.25), summed left to right), as the reference computes them.
int ps_build_pyramid(int device, const uint8_t* gray, uint32_t width, uint32_t height, const double* k,
                     uint32_t levels, uint8_t* const* out, uint32_t* out_w, uint32_t* out_h, double* out_k) {
  if (!gray || !out || !out_w || !out_h || levels < 1 || width < 1 || height < 1 || levels > 16) return PS_EINVAL;
  for (uint32_t i = 0; i < levels; ++i)
    if (!out[i]) return PS_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return PS_ENODEV;
  }
  const float e = std::exp(-1.0f / (2.0f * 0.25f));
  const float sum = (e + 1.0f) + e;
  const float g[3] = {e / sum, 1.0f / sum, e / sum};
  std::vector<uint32_t> w(levels), h(levels);  // finest first
  w[0] = width;
  h[0] = height;
  size_t total = 0;
  for (uint32_t i = 0; i < levels; ++i) {
    if (i) {
      w[i] = w[i - 1] / 2;
      h[i] = h[i - 1] / 2;
      if (w[i] < 1 || h[i] < 1) return PS_EINVAL;
    }
    total += (size_t)w[i] * h[i];
  }
  unsigned char* d = nullptr;
  cudaStream_t st = nullptr;
  int rc = PS_OK;
  if (cudaMalloc(&d, total) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    rc = PS_ENOMEM;
  } else {
    size_t off = 0;
    std::vector<size_t> offs(levels);
    for (uint32_t i = 0; i < levels; ++i) {
      offs[i] = off;
      off += (size_t)w[i] * h[i];
    }
    cudaError_t ce = cudaMemcpyAsync(d, gray, (size_t)width * height, cudaMemcpyHostToDevice, st);
    for (uint32_t i = 1; i < levels && ce == cudaSuccess; ++i)
      ce = ps_post::launch_pyramid(d + offs[i - 1], (int)w[i - 1], (int)h[i - 1], d + offs[i], g, st);
    for (uint32_t i = 0; i < levels && ce == cudaSuccess; ++i)  // out[0] = coarsest
      ce = cudaMemcpyAsync(out[levels - 1 - i], d + offs[i], (size_t)w[i] * h[i], cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) rc = PS_ECUDA;
  }
  if (st) cudaStreamDestroy(st);
  cudaFree(d);
  cudaGetLastError();
  double kk[4] = {k ? k[0] : 0.0, k ? k[1] : 0.0, k ? k[2] : 0.0, k ? k[3] : 0.0};
  for (uint32_t i = 0; i < levels; ++i) {
    out_w[levels - 1 - i] = w[i];
    out_h[levels - 1 - i] = h[i];
    if (out_k) memcpy(out_k + 4 * (levels - 1 - i), kk, sizeof kk);
    kk[0] = kk[0] * 0.5;
    kk[1] = kk[1] * 0.5;
    kk[2] = (kk[2] + 0.5) * 0.5 - 0.5;
    kk[3] = (kk[3] + 0.5) * 0.5 - 0.5;
  }
  return rc;
}

int ps_synchronize(ps_session* s) {
  return guard(s, [&] { sync(s); });
}

void* ps_session_stream(const ps_session* s) { return s ? (void*)s->st : nullptr; }

int ps_set_profiling(ps_session* s, uint32_t enable) {
  return guard(s, [&] {
    collect_events(s);
    s->profiling = enable != 0;
  });
}

int ps_kernel_stats(ps_session* s, uint32_t kind, double* total_ms, uint64_t* launches, uint64_t* ncc_windows) {
  return guard(s, [&] {
    if (kind >= PS_KERNEL_KINDS) fail(PS_EINVAL, "kernel kind out of range");
    collect_events(s);
    unsigned long long c[PS_KERNEL_KINDS];
    cuda_ok(cudaMemcpyAsync(c, s->counters, sizeof c, cudaMemcpyDeviceToHost, s->st), "read counters");
    sync(s);
    if (total_ms) *total_ms = s->kind_ms[kind];
    if (launches) *launches = s->kind_launches[kind];
    if (ncc_windows) *ncc_windows = c[kind];
  });
}

int ps_kernel_staged_stats(ps_session* s, uint32_t kind, uint64_t* stats) {
  return guard(s, [&] {
    if (kind >= PS_KERNEL_KINDS) fail(PS_EINVAL, "kernel kind out of range");
    if (!stats) fail(PS_EINVAL, "stats is NULL");
    unsigned long long c[PS_STAGE_STATS];
    cuda_ok(cudaMemcpyAsync(c, s->counters + PS_KERNEL_KINDS + PS_STAGE_STATS * kind, sizeof c,
                            cudaMemcpyDeviceToHost, s->st),
            "read counters");
    sync(s);
    for (int k = 0; k < PS_STAGE_STATS; ++k) stats[k] = c[k];
  });
}

int ps_reset_stats(ps_session* s) {
  return guard(s, [&] {
    collect_events(s);
    for (int k = 0; k < PS_KERNEL_KINDS; ++k) {
      s->kind_ms[k] = 0;
      s->kind_launches[k] = 0;
    }
    cuda_ok(cudaMemsetAsync(s->counters, 0, (1 + PS_STAGE_STATS) * PS_KERNEL_KINDS * sizeof(unsigned long long), s->st), "memset");
    sync(s);
  });
}

int ps_check_reciprocal(int device, int exp_lo, int exp_hi, uint64_t* mismatches, uint32_t* first_bad) {
  if (!mismatches || exp_lo < -126 || exp_hi > 127 || exp_lo > exp_hi) return PS_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return PS_ENODEV;
  unsigned long long* bad = nullptr;
  unsigned* first = nullptr;
  int rc = PS_OK;
  if (cudaMalloc(&bad, sizeof(unsigned long long)) != cudaSuccess || cudaMalloc(&first, 8 * sizeof(unsigned)) != cudaSuccess)
    rc = PS_ENOMEM;
  if (rc == PS_OK && (cudaMemset(bad, 0, sizeof(unsigned long long)) != cudaSuccess ||
                      cudaMemset(first, 0, 8 * sizeof(unsigned)) != cudaSuccess))
    rc = PS_ECUDA;
  if (rc == PS_OK && ps_parity::launch_rcp_check(exp_lo, exp_hi, bad, first, 0) != cudaSuccess) rc = PS_ECUDA;
  unsigned long long h = 0;
  unsigned f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (rc == PS_OK && (cudaMemcpy(&h, bad, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess ||
                      cudaMemcpy(f, first, sizeof f, cudaMemcpyDeviceToHost) != cudaSuccess))
    rc = PS_ECUDA;
  if (rc == PS_OK) {
    *mismatches = h;
    if (first_bad) memcpy(first_bad, f, sizeof f);
  }
  cudaFree(bad);
  cudaFree(first);
  cudaGetLastError();
  return rc;
}

int ps_measure_fp32_peak(int device, double* tflops) {
  if (!tflops) return PS_EINVAL;
  if (cudaSetDevice(device) != cudaSuccess) return PS_ENODEV;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return PS_ENODEV;
  float* out = nullptr;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return PS_ECUDA;
  const int blocks = prop.multiProcessorCount * 8, iters = 2048;
  int rc = PS_OK;
  cudaEvent_t a, b;
  if (cudaMalloc(&out, blocks * sizeof(float)) != cudaSuccess) rc = PS_ENOMEM;
  if (rc == PS_OK) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    for (int rep = 0; rep < 4 && rc == PS_OK; ++rep) {
      cudaEventRecord(a, st);
      if (ps_parity::launch_fp32_probe(out, blocks, iters, st) != cudaSuccess) rc = PS_ECUDA;
      cudaEventRecord(b, st);
      if (cudaEventSynchronize(b) != cudaSuccess) rc = PS_ECUDA;
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      if (rep > 0 && ms < best) best = ms;  // first launch is warm-up
    }
    const double flop = 2.0 * 8 * 16 * (double)iters * blocks * 256;
    *tflops = flop / (best * 1e-3) / 1e12;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  cudaFree(out);
  cudaStreamDestroy(st);
  cudaGetLastError();
  return rc;
}

}  // extern "C"
