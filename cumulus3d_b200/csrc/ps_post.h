// Device-side tables of the post-processing kernels (ps_post.cu) shared with the session runtime.
#pragma once
#include <cuda_runtime.h>

#include "ps_types.h"

#define PS_FUSE_MAX_OVERLAP 32  // overlap views checked per reference pixel (consistency_num_images and num_neighbors)

namespace ps_post {

// One view of a speckle launch: slot offset, size, first CTA, minimum component area ceil(w·h·frac).
struct SpkItem {
  long long off;
  int w, h, tile0, min_area;
};

struct SpkArgs {
  float4* plane;       // readout planes (nx, ny, nz, d), erased in place
  const float* cost;   // final matching costs
  int* parent;         // union-find parent per slot pixel (-1 = invalid)
  int* size;           // component size per root
  unsigned* lo;        // bisection bounds per small root (order-preserving cost keys)
  unsigned* hi;
  unsigned* cnt;
  unsigned long long* removed;
  unsigned long long* valid;  // k_count_valid: valid pixels of the items
  float rel, keep;
  int nitems;
  SpkItem items[PS_MAX_ITEMS];
};

// Camera and depth map of one view for fusion: world -> camera x_c = R x_w + t (R row-major), intrinsics k.
struct FuseView {
  double k[4];
  double r[9];
  double t[3];
  double baseline;       // representative baseline (median source-centre distance), 0 = unweighted
  const float* img;      // image plane (for the gray colour), row pitch `pitch` floats
  long long off;         // slot offset of the view's depth map
  int w, h, pitch;
  unsigned image_id;
  unsigned idbase;       // second pass: candidate number of the view's first pixel (prefix of the fused views' sizes)
  int nov;               // overlap views to check, in order
  int ov[PS_FUSE_MAX_OVERLAP];
};

struct FuseArgs {
  const FuseView* views;  // device table indexed by session view
  int v;                  // reference view of this launch
  const float4* plane;    // readout planes of the level (slot layout)
  const float* cost;
  unsigned char* marks;   // "used" marks per slot pixel
  int min_views, mark_used, mark_radius, inverse_variance;
  double sigma0, slope, depth_tol, cos_n, r2;
  float* pos;
  float* nrm;
  unsigned char* col;
  unsigned long long* key;
  unsigned char* nvis;
  unsigned short* vis;    // vis_stride entries per point (sorted contributing views)
  int vis_stride;
  unsigned long long* count;
  unsigned long long capacity;
  // second pass of leftover pixels (fusion.rs:540-627)
  unsigned char* consumed;          // first pass: reference and agreeing pixels of adopted points (NULL: not kept)
  unsigned* owner;                  // smallest candidate number claiming each slot pixel
  const unsigned long long* gkeys;  // spatial hash of first-pass points (gcap slots, 0 = empty)
  const unsigned* gheads;           // first point of each slot's chain (0xffffffff: none)
  const unsigned* gnext;            // next point of the same slot
  unsigned gcap, gpoints;           // gcap = 0: no distance test
  double gcell;                     // cell size = minimum distance
};

// Score fusion (fuse_scored, crates/dense/src/fusion_score.rs:196-435).  Candidates are appended in any order; each
// carries its candidate number gid = idbase + pixel, whose order is the output order, and its priority
// (~total_order(score) << 32) | (gid + 1), smaller first, so that score descends and ties go to (view, pixel) order.
#define PS_SCORE_FREE 0xffffffffffffffffull
#define PS_SCORE_LOCKED 0ull
struct ScoreArgs {
  const FuseView* views;  // camera, slot offset, candidate numbering and overlap list per session view
  int v;                  // reference view of a candidate launch
  const float4* plane;    // readout planes of the level (slot layout)
  const float* cost;
  int inverse_variance, mark_used;
  double sigma0, slope, depth_tol, cos_n, k_e, k_t, lambda, tau;
  // candidates (capacity entries)
  float* pos;
  float* nrm;
  unsigned char* col;
  unsigned long long* key;
  unsigned char* nvis;
  unsigned short* vis;
  int vis_stride;
  unsigned* gid;
  unsigned long long* prio;
  unsigned* pix;          // pix_stride slot pixels per candidate: its reference pixel, then its agreeing pixels
  unsigned char* npix;
  int pix_stride;
  unsigned char* state;   // 2 undecided, 1 adopted, 0 rejected
  unsigned long long* count;
  unsigned long long capacity;
  // adoption rounds (fusion_score.rs:352-414)
  unsigned long long* claim;  // per slot pixel: PS_SCORE_FREE, PS_SCORE_LOCKED or the smallest claiming priority
  const unsigned* active;     // undecided candidates of this round (*ncur of them)
  unsigned* next;             // undecided candidates after it (*nnext)
  unsigned* ncur;
  unsigned* nnext;
  unsigned long long* adopted;
};
// candidates of view A.v (one thread per pixel)
cudaError_t launch_score_candidates(const ScoreArgs& A, int w, int h, cudaStream_t st);
// active = 0 .. n-1, *ncur = n
cudaError_t launch_score_init(const ScoreArgs& A, unsigned n, cudaStream_t st);
// one adoption round over *ncur active candidates (three launches; `blocks` CTAs of 256 threads each)
cudaError_t launch_score_round(const ScoreArgs& A, int blocks, cudaStream_t st);

// Free-space visibility filter of a fused cloud (filter_visibility, crates/dense/src/visibility.rs:106-151).
#define PS_VIS_MAX_CHECK 64
struct VisArgs {
  const FuseView* views;        // camera and slot offset per session view
  const float4* plane;          // readout planes (depth = w)
  const unsigned char* used;    // per session view: fused
  const int* ovoff;             // full overlap list of view v: ovlist[ovoff[v] .. ovoff[v+1])
  const int* ovlist;
  int nviews;
  const float* pos;
  const unsigned char* nvis;
  const unsigned short* vis;
  int vis_stride;
  unsigned long long n, n1;     // points; the first n1 are from the first pass
  int limit, min_violations;
  double tau;
  unsigned char* keep;
  int masked;                   // 1: only points whose keep entry is set are tested (the others stay out, uncounted)
  unsigned long long* removed;  // [0]: first-pass points removed, [1]: second-pass points removed
};

// Bilateral smoothing of a fused cloud along its normals (smooth_along_normals, crates/dense/src/smooth.rs:143-220).
struct SmoothArgs {
  float* pos;                         // cloud positions (read)
  float* pos2;                        // next positions (written)
  const float* nrm;
  const unsigned char* keep;          // visibility mask (NULL: every point)
  const unsigned long long* key;      // point keys; with the pass they give the cloud order
  const unsigned* gid;                // candidate numbers (score fusion): the cloud order instead (NULL: keys)
  unsigned long long n, n1;           // points; the first n1 are from the first pass
  double r, r2, inv_2ss, inv_2sr, cos_n;
  unsigned long long* hkeys;          // cell table (cap slots, 0 = empty)
  unsigned* hcnt;
  unsigned* hstart;
  unsigned* hcur;
  unsigned cap;
  unsigned* list;                     // points grouped by cell, each group in cloud order
  unsigned* pslot;                    // cell slot of each point
  unsigned* total;
  int* flag;                          // set when a cell is out of range or the table is full
};
// one Jacobi pass: cells, grouping, ordering, and the moves into pos2
cudaError_t launch_smooth_pass(const SmoothArgs& A, cudaStream_t st);

// Median sampling of the ground sample distance (depth_gsd, fusion.rs:469-487), one CTA per view.
struct GsdView {
  long long off;       // slot offset of the view's readout planes
  long long soff;      // first sample slot
  int npix;
  double fx;
};

// Hole filling of one view's readout planes (fill_holes, crates/dense/src/postproc.rs:139-201).
struct FillArgs {
  float4* plane;    // the view's readout planes (nx, ny, nz, d), filled in place
  float* cost;      // the view's run costs in; filled pixels take their source pixel's cost
  const float* img; // the view's image plane, row pitch `pitch` floats (gray = round(255·value))
  float4* tplane;   // scratch per pixel: its fill (d = 0: none)
  float* tcost;
  unsigned long long* filled;
  double k[4];
  int w, h, pitch, maxd, step;
  float max_cost;
};
cudaError_t launch_fill_holes(const FillArgs& A, cudaStream_t st);

cudaError_t launch_speckles(const SpkArgs& A, int ntiles, cudaStream_t st, int* launches);
cudaError_t launch_count_valid(const SpkArgs& A, int ntiles, cudaStream_t st);
cudaError_t launch_fuse(const FuseArgs& A, int w, int h, cudaStream_t st);
// second pass: stage 1 (candidates claim their pixels) and stage 2 (owners of their reference pixel are emitted)
cudaError_t launch_fuse_second(const FuseArgs& A, int w, int h, int stage, cudaStream_t st);
cudaError_t launch_visibility(const VisArgs& A, cudaStream_t st);
// per view: every 97th valid depth in row-major order, then their median over fx (gsd[i]; NaN when the view has none)
cudaError_t launch_gsd(const float4* plane, const GsdView* views, int nviews, float* samples, unsigned* scount,
                       double* gsd, cudaStream_t st);
// spatial hash of `n` points (positions x,y,z) with cells of size `cell` into a table of `cap` slots (a power of 2)
cudaError_t launch_grid_insert(const float* pos, unsigned n, double cell, unsigned long long* keys, unsigned* heads,
                               unsigned* next, unsigned cap, int* overflow, cudaStream_t st);
cudaError_t launch_pyramid(const unsigned char* in, int w, int h, unsigned char* out, const float* g, cudaStream_t st);
// 8-bit image (w × h, tight rows) -> f32 plane rows of `pitch` floats through a 256-entry table.
// Output order of a fused cloud on the device.  Every kept point owns one cell of a grid of `cells` cells per pass,
// laid out in output order: consistency fusion: pass (first, second) × the fused views in ascending image id × the
// view's pixels row-major, which is ascending key within a pass; score fusion: its candidate number (one pass).  The
// exclusive prefix sum of the occupied cells is each point's output index.
struct CloudOrderArgs {
  unsigned long long n, count1;    // emitted points; the first count1 are the first pass
  unsigned long long cells;        // cells per pass
  const unsigned char* keep;       // per point 1 = kept (NULL: all)
  const unsigned* gid;             // score fusion: candidate number = cell (NULL: consistency fusion, cell from key)
  const unsigned long long* key;
  const unsigned* ids;             // consistency fusion: the fused views' image ids, ascending and distinct
  const unsigned long long* base;  // their first cell
  const int* width;                // their widths
  int nids;
  unsigned* rank;                  // passes·cells entries: occupancy, then exclusive ranks
  const float* pos;                // the cloud as emitted
  const float* nrm;
  const unsigned char* col;
  const unsigned char* nvis;
  const unsigned short* vis;
  int vis_stride;
  float* opos;                     // the cloud in output order (any of opos..ovis may be NULL)
  float* onrm;
  unsigned char* ocol;
  unsigned long long* okey;
  unsigned char* onvis;
  unsigned short* ovis;
  int ovis_stride;
};
cudaError_t launch_cloud_mark(const CloudOrderArgs& A, cudaStream_t st);
cudaError_t launch_cloud_scatter(const CloudOrderArgs& A, cudaStream_t st);
// In-place exclusive prefix sum of n unsigned ints; `tmp` holds scan_scratch(n) entries.
size_t scan_scratch(size_t n);
cudaError_t scan_exclusive(unsigned* data, size_t n, unsigned* tmp, cudaStream_t st);

cudaError_t launch_u8_plane(const unsigned char* in, int w, int h, const float* lut, float* out, int pitch,
                            cudaStream_t st);

}  // namespace ps_post
