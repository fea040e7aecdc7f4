// Device-side descriptor tables of the PatchStereo engine (plain structs shared by the kernels and the host
// runtime).  They play the role of the reference's LevelDesc / PairRec / LevelPair / ViewDesc / BatchItem / KParams
// (crates/cuda/src/kernels/patchmatch.cu:52-109), laid out for this engine: images are normalised f32 planes with a
// zero border instead of texture objects, and the batch table travels inside the kernel parameters.
#pragma once
#include <stdint.h>

#define PS_MAXSRC 32
#define PS_MAX_ITEMS 64  // views per launch (reference max_batch default, crates/cuda/src/patchmatch.rs:76)
#define PS_BORDER 2      // zero border (pixels) around every image plane: bilinear taps never need bounds checks

// Half-step CTA: 128 threads, 4 warps; a warp covers 16 active columns × 2 rows of a 32 × 8 pixel tile.
#define PS_HALF_NT 128
#define PS_HALF_PW 32
#define PS_HALF2_PW 16  // two lanes per pixel: a warp = 8 active columns × 2 rows × 2 lanes
#define PS_HALF_PH 8
// Staged-source half step (PS_TUNE_STAGED): a warp covers an 8 × 8 pixel block (4 active columns × 8 rows) of the
// 32 × 8 tile and stages the union of its lanes' source footprints of one window into a PS_BOX_P × PS_BOX_H box of
// shared memory.  The pitch is ≡ 4 (mod 16) so that the warp's ideal access pattern is free of bank conflicts.
#define PS_BOX_P 36
#define PS_BOX_H 32
// Reference tile pitch of the staged half step (≡ 4 mod 8: the warp's 8 × 8 block reads it without bank conflicts).
#define PS_HALF_ST_TW(wr) ((((PS_HALF_PW) + 2 * (wr) + 3) / 8) * 8 + 4)
#define PS_STAGE_MIN_LANES 4
#define PS_STAGE_STATS 8  // profiling counters of the staged half step per kernel kind
// Evaluate / filter CTA: 128 threads covering 32 × 4 pixels (a warp is one row).
#define PS_EVAL_NT 128
#define PS_EVAL_PW 32
#define PS_EVAL_PH 4
// Simple per-pixel kernels (upsample, median, readout, snapshot): 32 × 8 threads.
#define PS_SIMPLE_BX 32
#define PS_SIMPLE_BY 8
// Learned proposal: network input channels (image, PS_SWEEP_PLANES sweep costs, zero padding to a multiple of 16);
// the same values as the C ABI header.
#ifndef PS_SWEEP_PLANES
#define PS_SWEEP_PLANES 32
#endif
#ifndef PS_NET_CH_IN
#define PS_NET_CH_IN 48
#endif

// Bounds-checked build (ps_options.checked, namespace ps_checked): the kernels test the indices that come from data
// or from non-trivial arithmetic before they access memory.  A failed test skips the access and records the first
// violation in the launch's fault word as (site << 56) | (index mod 2^56); the runtime turns a non-zero word into
// PS_EFAULT.  Nothing traps.
enum PsCheckSite {
  PS_SITE_NONE = 0,
  PS_SITE_TILE = 1,      // reference tile in shared memory (window taps, reference statistics)
  PS_SITE_BOX = 2,       // staged source box in shared memory (the footprint bound)
  PS_SITE_PLANE = 3,     // bordered source plane in global memory (bilinear taps)
  PS_SITE_STATE = 4,     // per-pixel state arrays (plane, cost, best view, prior)
  PS_SITE_SOURCE = 5,    // source view index of a pair
  PS_SITE_SNAPSHOT = 6,  // depth snapshot of a source view (geometric term)
  PS_SITE_PROBE = 7,     // self-test: one deliberately out-of-range index, evaluated when PsRun.probe is set
};

// One (view, level) image plane.
struct PsLevel {
  const float* img;    // pixel (0,0) of a plane with PS_BORDER zero rows/columns on every side
  unsigned long long tex;  // border-addressed point texture of the same plane (cudaTextureObject_t), 0 if not built
  int w, h, pitch;         // pitch in floats
  int pad;
  float fx, fy, cx, cy;
};

// Reference -> source relative geometry (PairGeometry) plus the source view index.
struct PsPair {
  float r[9];
  float t[3];
  float c[3];
  int src;
};

// Constant part of the plane-induced homography at one level: A = K_j R K^-1, b = K_j t.
struct PsLPair {
  float A[9];
  float b[3];
};

struct PsView {
  unsigned long long key;
  float dmin, dmax;
  int nsrc, pad;
};

// One view of a launch.  `off` indexes the per-pixel state arrays of the view's level slot; `aux` is the offset of
// the view's low-level planes for upsampling; `tile0` is the first CTA of this item (prefix sum over items).
struct PsItem {
  long long off;
  long long aux;
  int view, w, h, tile0;
};

// Persistent half-step kernel (PS_TUNE_PERSISTENT): one launch runs every half step of a run (up to PS_MAX_PHASES
// of them) over a device work queue of (phase, tile) items; a tile of phase k waits, with a bounded spin, until every
// tile of phase k - 1 of its view is done.  PS_QUEUE_SPIN_LIMIT polls (about a second with the back-off) end a wait
// with an error word that the runtime reports as PS_ETIMEOUT.
#define PS_MAX_PHASES 64
#define PS_QUEUE_SPIN_LIMIT (1u << 22)
struct PsPhase {
  int t, color;
  float tau_good, eps, phi;
};

// Launch parameters (kernel parameter space, so the batch table needs no device allocation).
struct PsRun {
  unsigned long long seed;
  const PsLevel* lv;
  const PsPair* pairs;
  const PsLPair* lpairs;
  const PsView* views;
  const float* snap;
  const long long* snap_off;
  float4* plane;
  float* cost;
  unsigned char* bview;
  unsigned char* count;
  const float4* prior;  // coarse-scale candidates (run) or low-level planes (upsample) or input planes (median)
  int nlevels, level, geometric, run_id;
  int t, color, random_init, topk;
  int use_prior, nitems, ntiles, maxsrc;
  int wr, ws;  // runtime window for the generic kernels
  float tau_good, tau_bad, inv2beta2, prev_w;
  int n1, n2;
  float inv2s, inv2c;
  float cos_tri_min, inv2inc, lambda, gmax;
  float eps, phi;
  float cos_filter_tri, q_min, ncc_norm, inv2ncc;
  float filter_gmax, weak_var;
  float up_inv2s, up_inv2c;  // joint bilateral upsampling constants
  int need_min;              // readout threshold: min_num_consistent
  int mode;                  // evaluate: 1 = run start (init + cost + clear best view), 0 = cost only
  unsigned long long* ncc_count;  // when set, kernels add the number of NCC window evaluations they performed
  unsigned long long* stage_count;  // when set (staged half step): PS_STAGE_STATS counters, see ps_kernel_staged_stats
  unsigned long long* fault;  // checked build: first failed bounds test (see PsCheckSite), 0 while none
  long long state_pixels;     // checked build: pixels of the state arrays the launch addresses (bound of off + pixel)
  long long snap_pixels;      // checked build: floats of the depth snapshot buffer
  int nviews_all;             // checked build: views of the session (bound of source view indices)
  int probe;                  // checked build: test one index past the end of the state arrays (self-test)
  const float4* proposal;  // run start with random init: planes with d > 0 replace the random draw (learned init)
  unsigned short* netin;   // plane sweep: bf16 network input [rows][netin_pitch][PS_NET_CH_IN] of the run's one view
  int netin_pitch;         // pixels per row of netin
  int sweep_ws;            // plane sweep: window step
  float sweep_n[3];        // plane sweep: plane normal in the reference camera frame (n · ray < 0)
  // persistent half step: queue[0] = next item, queue[1] = error word (a wait ran out), queue[2 + k·nitems + i] =
  // tiles of item i done in phase k; qstall (tests only) makes every wait need one tile more than exists
  unsigned* queue;
  int nphases, qstall;
  // TMA staging (PS_TUNE_TMA with PS_TUNE_STAGED): two 128-byte tensor maps per (view, level) plane, see tmap()
  const void* tmaps;
  PsItem items[PS_MAX_ITEMS];
  PsPhase phases[PS_MAX_PHASES];
};
