/*
 * patchstereo.h — C ABI of the B200 PatchStereo depth-map engine (libpatchstereo.so).
 *
 * The engine is a drop-in for the PatchMatch backend that cumulus3d-dense drives through cumulus3d-cuda.  Each
 * entry point below replaces one method of the reference's Rust traits; the reference file:line is given beside it
 * (paths inside the cumulus3d project):
 *
 *   trait PatchMatchBackend  crates/dense/src/kernel.rs:240-245   (impl CudaPatchMatch crates/cuda/src/patchmatch.rs:285-298)
 *   trait PatchMatchSession  crates/dense/src/kernel.rs:192-237   (impl Session crates/cuda/src/patchmatch.rs:751-869)
 *
 * Conventions (same as the reference, crates/dense/src/kernel.rs:36-74): an integer pixel index is the pixel
 * centre; ray(x,y) = ((x-cx)/fx, (y-cy)/fy, 1); depth is camera z; normals are unit vectors in reference-camera
 * coordinates with n·ray < 0.  Level 0 is the coarsest scale.
 *
 * All pointers are borrowed: the caller owns them and they only need to stay valid for the duration of the call
 * (ps_begin copies every image and geometry table to the device).  No call allocates memory the caller must free.
 * Every entry point returns a ps_status; the message of the last failure is available from ps_last_error /
 * ps_backend_last_error.  No C++ exception crosses this boundary.
 *
 * Threading: a backend serialises sessions (one open session per backend at a time, as the reference's mutex in
 * crates/cuda/src/patchmatch.rs:96-97).  A session owns one CUDA stream and is not thread-safe.  Blocking calls
 * return after their results are in host memory.
 */
#ifndef PATCHSTEREO_H
#define PATCHSTEREO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PS_MAX_SOURCES 32 /* crates/cuda/src/kernels/patchmatch.cu:40 (MAXSRC) */
#define PS_ABI_VERSION 5

/* Status codes.  Maps the reference's error kinds: Error::InvalidArgument -> PS_EINVAL,
 * Error::Invariant("CUDA: …") -> PS_ECUDA (crates/cuda/src/patchmatch.rs:234-236),
 * GpuError::NotAvailable -> PS_ENODEV (crates/cuda/src/device.rs:190-201). */
typedef enum ps_status {
  PS_OK = 0,
  PS_EINVAL = 1,   /* bad argument, size or parameter */
  PS_ECUDA = 2,    /* CUDA runtime / driver failure */
  PS_ENODEV = 3,   /* no usable sm_100 device */
  PS_ECOMPILE = 4, /* unused: kernels are compiled ahead of time for sm_100a */
  PS_ETIMEOUT = 5, /* a bounded device-side wait gave up */
  PS_EFAULT = 6,   /* a checked build detected an out-of-bounds index */
  PS_ENOMEM = 7,   /* device or pinned allocation failed */
  PS_EBUSY = 8     /* the backend already has an open session */
} ps_status;

typedef enum ps_image_format {
  PS_IMAGE_U8 = 0,  /* 8-bit gray, value/255 (crates/dense/src/kernel.rs:87-88, patchmatch.cu:141) */
  PS_IMAGE_F32 = 1  /* 32-bit float gray, used as is (intended range [0,1]) */
} ps_image_format;

typedef enum ps_math_mode {
  PS_MATH_PARITY = 0, /* IEEE division/sqrt, the project's own exp/sincos, explicit fma: bitwise equal to the oracle */
  PS_MATH_FAST = 1    /* hardware approximate reciprocal/exp/rsqrt (the reference's "speed first" numerics) */
} ps_math_mode;

/* Backend options (cf. CudaPatchMatchOptions, crates/cuda/src/patchmatch.rs:56-81). */
typedef struct ps_options {
  uint32_t math_mode;    /* ps_math_mode */
  uint32_t max_batch;    /* views per launch; 0 = 64 (reference default) */
  uint64_t batch_pixels; /* pixel budget per launch; 0 = unbounded (HBM holds every view of a job) */
  uint32_t checked;      /* 1 = bounds-checked kernels (parity math; not with PS_MATH_FAST): every data-dependent index
                            is tested before its access, a failed test skips the access and the next synchronising
                            call fails with PS_EFAULT naming the first violation; the results are those of the parity
                            build.  The half step, evaluate, filter, upsample, median, readout and snapshot kernels are
                            checked; post-processing, fusion, neighbours and the network are not. */
  uint32_t tuning;       /* half-step kernel variant, PS_TUNE_* flags; 0 = defaults (the autotuner sets these) */
} ps_options;

/* Half-step kernel variants (same results bit for bit; only speed differs). */
#define PS_TUNE_NO_WEIGHT_CACHE 0x1u /* recompute window weights per tap (more CTAs per SM, more exp work) */
#define PS_TUNE_TEX_GATHER 0x2u      /* fetch each bilinear 2×2 footprint with one texture gather (same bits) */
#define PS_TUNE_ONE_LANE 0x4u        /* one thread per pixel (default: two lanes per pixel split the window rows) */
#define PS_TUNE_ROW_PAIRS 0x8u       /* one thread per pixel, window rows 2p and 2p+1 as packed f32x2 pairs */
#define PS_TUNE_STAGED 0x10u         /* row pairs, and each warp stages its sources' footprints in shared memory */
#define PS_TUNE_PERSISTENT 0x20u     /* with PS_TUNE_ROW_PAIRS: one persistent launch per run over a device work queue of
                                        (half step, tile) items with bounded per-view waits between half steps; a
                                        wait that gives up fails the call with PS_ETIMEOUT */
#define PS_TUNE_TMA 0x40u            /* with PS_TUNE_STAGED: the reference tile and the source boxes arrive by 2-D TMA
                                        tensor loads (cp.async.bulk.tensor, no multicast) on mbarriers */
#define PS_TUNE_VALID_MASK 0x7Fu

/* PmParams (crates/dense/src/params.rs:76-124, defaults :126-154). */
typedef struct ps_pm_params {
  int32_t window_radius;
  int32_t window_step;
  float sigma_spatial; /* <= 0: window radius (PmParams::sigma_s, params.rs:158-164) */
  float sigma_color;
  float tau0;
  float tau_alpha;
  float tau1;
  float beta;
  uint32_t n1;
  uint32_t n2;
  float prev_view_weight;
  float min_triangulation_angle_deg;
  float incident_angle_sigma;
  float geom_lambda;
  float geom_max_cost;
  uint32_t top_k;
  float eps0_photometric;
  float eps0_geometric;
  float phi0_photometric_deg;
  float phi0_geometric_deg;
  float eps_min;
  float phi_min_deg;
  float weak_texture_var;
} ps_pm_params;

/* FilterParams (crates/dense/src/params.rs:180-207). */
typedef struct ps_filter_params {
  float min_ncc;
  float min_triangulation_angle_deg;
  uint32_t min_num_consistent;
  float geom_max_cost;
  float ncc_sigma;
  uint32_t median_filter;
} ps_filter_params;

/* LevelImage (crates/dense/src/kernel.rs:80-91), with a pixel format added for float inputs. */
typedef struct ps_level_image {
  uint32_t width;
  uint32_t height;
  uint32_t format;    /* ps_image_format */
  uint32_t stride;    /* elements per row; 0 = width */
  const void* pixels; /* row-major */
  float k[4];         /* fx, fy, cx, cy (integer-centre convention) */
} ps_level_image;

/* PairGeometry (crates/dense/src/kernel.rs:93-103), same repr(C) layout. */
typedef struct ps_pair_geometry {
  float r[9];      /* reference -> source rotation, row-major */
  float t[3];      /* reference -> source translation */
  float center[3]; /* source centre in reference-camera coordinates */
} ps_pair_geometry;

/* KernelView (crates/dense/src/kernel.rs:105-120). */
typedef struct ps_kernel_view {
  uint64_t key;                   /* RNG key, FNV-1a of the image name (crates/dense/src/math.rs:31-39) */
  const ps_level_image* levels;   /* num_levels entries, 0 = coarsest */
  const uint32_t* sources;        /* num_sources view indices (<= PS_MAX_SOURCES) */
  uint32_t num_sources;
  uint32_t reserved;
  const ps_pair_geometry* pairs;  /* num_sources entries */
  const double* pairs_f64;        /* optional: num_sources × 15 doubles (r[9], t[3], center[3]); when given, the
                                     homography setup A = K_j R K^-1, b = K_j t runs from these in FP64 */
  float depth_min;
  float depth_max;
} ps_kernel_view;

/* KernelInput (crates/dense/src/kernel.rs:122-135). */
typedef struct ps_kernel_input {
  const ps_kernel_view* views;
  uint32_t num_views;
  uint32_t num_levels;
  ps_pm_params pm;
  ps_filter_params filter;
  uint64_t seed;
} ps_kernel_input;

/* ViewState (crates/dense/src/kernel.rs:137-160): caller-owned arrays, updated in place by ps_run. */
typedef struct ps_view_state {
  uint32_t width;
  uint32_t height;
  float* depth;       /* w*h */
  float* normal;      /* 3*w*h, xyz interleaved */
  float* cost;        /* w*h */
  const float* prior; /* 4*w*h (nx,ny,nz,d) or NULL (= empty) */
} ps_view_state;

/* RunParams (crates/dense/src/kernel.rs:173-189).  random_init: 0 = keep the states' planes, PS_INIT_RANDOM = seeded
 * random planes (the reference's `true`), PS_INIT_PROPOSAL = the session's learned proposal where one exists and the
 * same random draw elsewhere (no reference counterpart; see ps_propose). */
#define PS_INIT_RANDOM 1u
#define PS_INIT_PROPOSAL 2u
typedef struct ps_run_params {
  uint32_t level;
  uint32_t geometric;
  uint32_t random_init;
  uint32_t iterations;
  uint32_t run_id;
  uint32_t use_prior;
} ps_run_params;

/* DepthSnapshot (crates/dense/src/kernel.rs:162-171): maps[v] is the depth map of view v at `level`
 * (width*height floats) or NULL when absent.  Equal id implies equal content. */
typedef struct ps_depth_snapshot {
  uint64_t id;
  uint32_t level;
  uint32_t num_maps;
  const float* const* maps;
  /* optional (NULL = every map has its level's width*height elements): the element count of every map; a map whose
   * count differs from its level's width*height is left out of the snapshot, as the reference leaves it out
   * (crates/cuda/src/patchmatch.rs:573-604, the Vec lengths of DepthSnapshot::maps) */
  const uint64_t* map_lengths;
} ps_depth_snapshot;

typedef struct ps_backend ps_backend;
typedef struct ps_session ps_session;

/* ---- host-side failure injection (no counterpart in the reference; for tests of the error paths) ----------
 * Arms one failure on the backend: after `after` more operations of `kind` succeed, the next one fails as a device
 * would (PS_INJECT_DEVICE_ALLOC: a device allocation, reported as PS_ENOMEM; PS_INJECT_UPLOAD: a host-to-device copy
 * of images, states or snapshots, reported as PS_ECUDA), then the injection disarms itself.  PS_INJECT_NONE disarms.
 * Nothing reaches the GPU: the failing operation is refused on the host before it is issued. */
#define PS_INJECT_NONE 0u
#define PS_INJECT_DEVICE_ALLOC 1u
#define PS_INJECT_UPLOAD 2u
/* Checked backends only: the kernels launched until the next synchronising call each test one index past the end of
 * the state arrays (the test fails, no access is made), so that call fails with PS_EFAULT ("self-test probe"); the
 * probe is then spent.  Captured schedules (CUDA graphs) do not carry it.  `after` is ignored. */
#define PS_INJECT_CHECK_PROBE 3u
/* Persistent half step (PS_TUNE_PERSISTENT): the launches until the next synchronising call make every wait of their
 * queue need one tile more than exists, so the first wait runs out its bounded spin (about a second), the others
 * return at once, and that call fails with PS_ETIMEOUT; the stall is then spent.  Not carried by captured schedules.
 * `after` is ignored. */
#define PS_INJECT_QUEUE_STALL 4u
int ps_backend_inject_failure(ps_backend* be, uint32_t kind, uint32_t after);

/* ---- defaults and diagnostics ------------------------------------------------------------------------------ */
int ps_abi_version(void);
void ps_pm_params_default(ps_pm_params* out);         /* PmParams::default, crates/dense/src/params.rs:126-154 */
void ps_filter_params_default(ps_filter_params* out); /* FilterParams::default, crates/dense/src/params.rs:196-207 */
void ps_options_default(ps_options* out);             /* CudaPatchMatchOptions::default, patchmatch.rs:71-81 */

/* ---- PatchMatchBackend ------------------------------------------------------------------------------------- */
/* CudaPatchMatch::new / try_default (crates/cuda/src/patchmatch.rs:238-246).  A backend runs one session at a time
 * and keeps what its last session used for the next one: device buffers (a stream-ordered memory pool that does not
 * release freed memory), the pinned host staging buffer and the texture arrays.  ps_backend_destroy releases them;
 * end the backend's session first. */
int ps_backend_create(int device, const ps_options* opts, ps_backend** out);
void ps_backend_destroy(ps_backend* be);
/* PatchMatchBackend::name (crates/dense/src/kernel.rs:241-242); the string lives as long as the backend. */
const char* ps_backend_name(const ps_backend* be);
const char* ps_backend_last_error(const ps_backend* be);
/* PatchMatchBackend::begin (crates/dense/src/kernel.rs:243-244; crates/cuda/src/patchmatch.rs:289-297, Session::new
 * :355-547): validates, uploads every level of every view, builds the FP64 homography tables. */
int ps_begin(ps_backend* be, const ps_kernel_input* input, ps_session** out);
/* Drop for Session (crates/cuda/src/patchmatch.rs:992-1009): frees the device state, releases the backend. */
int ps_end(ps_session* s);
const char* ps_last_error(const ps_session* s);

/* ---- PatchMatchSession ------------------------------------------------------------------------------------- */
/* PatchMatchSession::run (crates/dense/src/kernel.rs:193-194; crates/cuda/src/patchmatch.rs:752-799).  A geometric
 * run requires a snapshot. */
int ps_run(ps_session* s, const uint32_t* views, size_t n, ps_view_state* states, const ps_run_params* p,
           const ps_depth_snapshot* snapshot);
/* PatchMatchSession::evaluate (crates/dense/src/kernel.rs:195-203; patchmatch.rs:801-824): out_cost[i] receives
 * w*h floats for views[i]. */
int ps_evaluate(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_view_state* states,
                uint32_t geometric, const ps_depth_snapshot* snapshot, float* const* out_cost);
/* PatchMatchSession::filter (crates/dense/src/kernel.rs:204-207; patchmatch.rs:842-868): out_counts[i] receives
 * w*h bytes. */
int ps_filter(ps_session* s, const uint32_t* views, size_t n, const ps_view_state* states,
              const ps_depth_snapshot* snapshot, uint8_t* const* out_counts);
/* PatchMatchSession::upsample (crates/dense/src/kernel.rs:208-232; patchmatch.rs:826-836, :931-960): low[i] is at
 * level-1, out[i] (caller-allocated depth/normal/cost at `level`) receives the upsampled planes, cost = 2. */
int ps_upsample(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_view_state* low,
                float sigma_s, float sigma_c, ps_view_state* out);
/* PatchMatchSession::median_filter (crates/dense/src/kernel.rs:233-236; patchmatch.rs:838-840, :962-989). */
int ps_median_filter(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_view_state* in,
                     ps_view_state* out);

/* ---- device-resident extension (no reference counterpart: the reference re-uploads states per call) --------
 * The session keeps one state slot per (view, level) in HBM.  These calls let a caller run the whole schedule
 * without host round trips; ps_run/ps_evaluate/ps_filter above are implemented on top of them. */
int ps_state_upload(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_view_state* states);
int ps_state_download(ps_session* s, uint32_t level, const uint32_t* views, size_t n, ps_view_state* states);
int ps_run_resident(ps_session* s, const uint32_t* views, size_t n, const ps_run_params* p);
/* Copies the resident depth of `views` at `level` into the session's snapshot buffer (other views become absent
 * unless `keep_others`). */
int ps_snapshot_capture(ps_session* s, uint32_t level, const uint32_t* views, size_t n, uint64_t id,
                        uint32_t keep_others);
/* The snapshot buffer of `level` in device memory (allocated on first use), laid out like the level's state slots:
 * offsets[v] (num_views entries, in floats) is where view v's w*h depth map lives.  A multi-GPU caller writes the
 * maps of views owned by other ranks there (e.g. NCCL broadcast into this GPU's own memory) and then declares them
 * with ps_snapshot_mark. */
int ps_snapshot_buffer(ps_session* s, uint32_t level, float** device_ptr, uint64_t* offsets);
/* Declares the maps of `views` present in the snapshot buffer of `level` (content written by the caller) and sets
 * the snapshot id; views not listed keep their current presence. */
int ps_snapshot_mark(ps_session* s, uint32_t level, const uint32_t* views, size_t n, uint64_t id);
/* Filter on the resident states against the resident snapshot; out_counts may be NULL (counts stay on device and
 * ps_readout_resident applies the threshold). */
int ps_filter_resident(ps_session* s, const uint32_t* views, size_t n, uint8_t* const* out_counts);
/* Readout threshold of crates/dense/src/densify.rs:441-454 on device: depth and normal are zeroed where
 * count < max(1, min(min_num_consistent, nsrc)); writes the result into out (host) when given. */
int ps_readout_resident(ps_session* s, const uint32_t* views, size_t n, ps_view_state* out);
/* A whole single-level schedule on resident states: photometric run (random init), `geometric_rounds` geometric runs
 * each against a snapshot of `views` captured on the device, the filter against a final snapshot and the readout
 * threshold (results stay resident).  With `use_graph`, the sequence is captured once into a CUDA graph per
 * (views, schedule, profiling flag) and replayed with one cudaGraphLaunch per call: no host synchronisation and no
 * host copies inside.  Asynchronous: returns after enqueueing; ps_synchronize waits.  No reference counterpart (the
 * reference drives every run from the host, crates/dense/src/densify.rs:351-439). */
typedef struct ps_schedule {
  uint32_t level;
  uint32_t photometric_iters;
  uint32_t geometric_rounds;
  uint32_t geometric_iters;
  uint32_t run_id_base; /* run ids run_id_base, run_id_base+1, … (RNG keys) */
  uint32_t use_graph;
  uint32_t init; /* initialisation of the photometric run: PS_INIT_RANDOM or PS_INIT_PROPOSAL */
} ps_schedule;
int ps_schedule_resident(ps_session* s, const uint32_t* views, size_t n, const ps_schedule* sch);
/* The multi-scale driver of compute_depth_maps (crates/dense/src/densify.rs:350-454, restorer without random init)
 * on resident states over every level of the session, captured into one CUDA graph per (views, schedule, profiling
 * flag) when use_graph: coarsest level from random init; each finer level upsampled (JBU), evaluated, refined by a
 * restorer run from the upsampled planes, evaluated again and merged per pixel (the restorer's plane where the
 * upsampled one is invalid or its cost exceeds the restorer's by more than restorer_threshold); geometric rounds at
 * every level against device-captured snapshots; at the top level the median filter (when the filter parameters enable
 * it), the filter and the readout threshold (results in the top level's readout planes).  Asynchronous.  No reference
 * counterpart (the reference drives these steps from the host). */
typedef struct ps_multiscale_schedule {
  uint32_t photometric_iters;       /* coarsest level (6) */
  uint32_t photometric_iters_upper; /* finer levels (3) */
  uint32_t geometric_rounds;        /* per level (2) */
  uint32_t geometric_iters;         /* (2) */
  float jbu_sigma_spatial;          /* 1.0 */
  float jbu_sigma_color;            /* 0.04 */
  float restorer_threshold;         /* 0.1 */
  uint32_t weak_texture_prior;      /* upsampled planes as the coarse prior of finer levels (0) */
  uint32_t run_id_base;             /* 1 */
  uint32_t use_graph;               /* 1 */
} ps_multiscale_schedule;
void ps_multiscale_schedule_default(ps_multiscale_schedule* out);
int ps_schedule_multiscale(ps_session* s, const uint32_t* views, size_t n, const ps_multiscale_schedule* m);
int ps_synchronize(ps_session* s);
/* Number of kernel launches this session issued so far (for launch accounting). */
uint64_t ps_launch_count(const ps_session* s);
/* The session's CUDA stream (a cudaStream_t), for callers that record their own events on it. */
void* ps_session_stream(const ps_session* s);

/* ---- allocation-free median filter (no counterpart in the reference) ---------------------------------------
 * For callers that own device buffers but may not allocate device memory (a host framework's memory pool owns every
 * allocation, a fixed budget forbids growth after start-up, or a real-time loop must not allocate).  Filters the
 * caller's planes in place: `planes` is device (or managed) memory of `device`, 16-byte aligned, width*height float4
 * (nx, ny, nz, d), and k = fx, fy, cx, cy of the image; other pointers are rejected with PS_EINVAL before any device
 * work.  Same rule as ps_median_filter, and the same bits as the median filter of a parity-math session.  Instead of
 * a session buffer, the input copy lives in a static device array of PS_NOALLOC_MAX_PIXELS planes (32 MiB, reserved
 * on every GPU that loads the library until exit); larger images are rejected with PS_EINVAL.  No cudaMalloc or
 * cudaFree is called.  All calls on a device share that array and it keeps the last call's contents (a call reads
 * only what it copied, so nothing needs clearing); calls that overlap on the GPU race on it.  The first call on a
 * device looks up the array's address with that device current; make it before any stream capture; the address is
 * kept, so it is stale after the caller resets that device.  The caller's current device is restored before the
 * call returns.  While the calling thread has a CUDA error pending the call does nothing and returns PS_ECUDA,
 * leaving that error pending.  Asynchronous on `stream` (a cudaStream_t, NULL = default stream). */
#define PS_NOALLOC_MAX_PIXELS (1u << 21)
int ps_median_filter_inplace_noalloc(int device, float* planes, uint32_t width, uint32_t height, const float* k,
                                     void* stream);

/* ---- learned proposal (no counterpart in the reference) -----------------------------------------------------
 * A BF16 encoder-decoder network predicts an initial plane and a confidence per pixel from the reference image and a
 * plane-sweep cost volume.  A run start with random_init = PS_INIT_PROPOSAL takes the proposed plane where the
 * confidence reached the threshold and the ordinary random draw everywhere else, so plain random initialisation is
 * the per-pixel fallback.
 * Network tensors are NHWC in device memory with height and width multiples of 8: input bf16 (raw bits)
 * [batch][height][width][PS_NET_CH_IN] = (image, PS_SWEEP_PLANES sweep costs, zeros); output f32
 * [batch][height][width][PS_NET_CH_OUT] = (logit of t = (1/d - 1/dmax) / (1/dmin - 1/dmax), normal xyz (not unit),
 * logit of the confidence, 3 unused).  Parameters: 12 convolutions 3×3 in the order e0a e0b e1a e1b e2a e2b e3a e3b d2
 * d1 d0 head with (cin, cout) = (48,32) (32,32) (32,64) (64,64) (64,96) (96,96) (96,128) (128,128) (224,96) (160,64)
 * (96,32) (32,8); each stores W [cout][9][cin] (tap = 3·(dy+1) + (dx+1)) then b [cout], f32.  A net is not
 * thread-safe. */
#define PS_SWEEP_PLANES 32
#define PS_NET_CH_IN 48
#define PS_NET_CH_OUT 8
typedef struct ps_net ps_net;
/* Seeded He-uniform initialisation on `device`. */
int ps_net_create(int device, uint64_t seed, ps_net** out);
void ps_net_destroy(ps_net* net);
const char* ps_net_last_error(const ps_net* net);
uint64_t ps_net_num_params(const ps_net* net);
uint32_t ps_net_step(const ps_net* net); /* AdamW steps taken */
int ps_net_get_params(ps_net* net, float* host);       /* num_params floats */
int ps_net_set_params(ps_net* net, const float* host); /* also resets nothing of the optimiser state */
/* Forward on device buffers, enqueued on `stream` (a cudaStream_t; NULL = the net's own stream, then blocking). */
int ps_net_forward(ps_net* net, const void* input, uint32_t batch, uint32_t height, uint32_t width, float* out,
                   void* stream);
/* One AdamW step (β = 0.9, 0.999, ε = 1e-8; weight decay on weights only) on device buffers: labels f32
 * [batch][height][width][6] = (t*, normal xyz, valid, depth d*).  Loss per valid pixel |σ(o0) - t*| + (1 - n̂·n*) +
 * 0.5·BCE(σ(o4), |d - d*| < 0.01·d*), averaged.  lr = 0 computes the loss and gradients only.  grad_out (host,
 * num_params floats, may be NULL) receives the gradients.  Blocking. */
int ps_net_train_step(ps_net* net, const void* input, const float* labels, uint32_t batch, uint32_t height,
                      uint32_t width, float depth_min, float depth_max, float lr, float weight_decay, float* loss,
                      float* grad_out);
/* Convolution kernels of every net in the process: 0 (default) = tcgen05 (5th-generation tensor cores,
 * tensor-memory accumulators) for cout in {64, 96, 128} and mma.sync otherwise; 1 = mma.sync only; 2 = tcgen05 for
 * every cout in {32, 64, 96, 128}. */
int ps_net_set_conv_path(int path);
/* Bounded waits of the tcgen05 convolution that expired on `device` (its results are then invalid); reset clears. */
int ps_net_conv_timeouts(int device, uint32_t* count, int reset);
/* Failure test of the bounded waits (on = 1): the tensor-core convolution's issuing thread stops committing work, so
 * its waits expire, it records the failure and returns; clear with on = 0 and reset the counter afterwards. */
int ps_net_test_stall_convolutions(int device, int on);
/* One 3×3 convolution (no bias) on host buffers through the network's kernels, for gradient checks: y = conv(x, w),
 * dx = conv(dy, flipped wᵀ), dw = Σ dy ⊗ im2col(x).  x, dy: bf16 bits NHWC; w f32 [cout][9][cin] (rounded to bf16);
 * cin and cout multiples of 8. */
int ps_net_conv_check(int device, const uint16_t* x, const float* w, const uint16_t* dy, uint32_t batch,
                      uint32_t height, uint32_t width, uint32_t cin, uint32_t cout, float* y, float* dx, float* dw);
/* Network input of one view at `level` into device memory `out` (rows of `row_pixels` >= width pixels; the caller
 * zeroes any padding): the image and PS_SWEEP_PLANES fronto-parallel plane-sweep NCC costs (inverse depths at bin
 * centres between 1/dmax and 1/dmin; mean over the first two sources; window radius as the session's, step 2).
 * Asynchronous on the session stream. */
int ps_sweep_volume(ps_session* s, uint32_t level, uint32_t view, void* out, uint32_t row_pixels);
/* Plane normal of each view's sweep in its camera frame (3 floats per session view; NULL = fronto-parallel
 * (0, 0, -1), the default).  Aerial callers pass the world's up direction seen from the camera (R · up), so the sweep
 * planes follow the ground's tilt.  Unit length, z < 0. */
int ps_set_sweep_normals(ps_session* s, const float* normals);
/* Sweep + network + decode for `views` at `level`: stores each view's proposal (planes with d = 0 where the
 * confidence is below conf_threshold) in the session for a later PS_INIT_PROPOSAL run start.  `proposed` (may be
 * NULL; then asynchronous) receives the number of proposed pixels; with it the call also fails with PS_ETIMEOUT if a
 * bounded wait of the tensor-core convolution expired (ps_net_conv_timeouts). */
int ps_propose(ps_session* s, ps_net* net, uint32_t level, const uint32_t* views, size_t n, float conf_threshold,
               uint64_t* proposed);
/* Caller-supplied proposals (host, 4·w·h floats (nx, ny, nz, d), d <= 0 = none) and read-back of the stored ones
 * (conf may be NULL). */
int ps_proposal_upload(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const float* const* planes);
int ps_proposal_download(ps_session* s, uint32_t level, const uint32_t* views, size_t n, float* const* planes,
                         float* const* conf);

/* ---- post-processing and fusion of resident depth maps -------------------------------------------------------
 * PostParams (crates/dense/src/postproc.rs:41-74), applied to the readout planes of `level` in place, in the
 * reference's order (crates/dense/src/densify.rs:455-461):
 *  - remove_speckles (postproc.rs:77-129): 4-connected components (|d_j - d_i| <= rel·min(d_i, d_j)) smaller than
 *    ceil(w·h·min_area_frac) whose lower median cost exceeds keep_cost are erased;
 *  - fill_holes (postproc.rs:139-201, off by default): every invalid pixel whose run cost is at most fill_max_cost
 *    walks the 8 directions up to round(diag·fill_max_frac) steps over the 8-bit gray image, stopping where the gray
 *    value jumps by more than fill_edge_step·255, and takes the plane of the valid pixel it meets with the smallest
 *    (gray difference, distance); filled pixels also take that pixel's cost (the slot's costs then hold the readout
 *    costs, as DepthMapResult.cost does).  The gray value of a pixel is round(255·plane value), which is the 8-bit
 *    input exactly for 8-bit images.  `intrinsics` (4 doubles fx, fy, cx, cy per session view, indexed by view;
 *    may be NULL) gives the full-precision DenseView::k the reference's rays use; NULL uses the level's.
 * Asynchronous unless `removed` / `filled` is given (then it receives the count). */
typedef struct ps_post_params {
  uint32_t remove_speckles;     /* true */
  float speckle_rel_depth;      /* 0.02 */
  double speckle_min_area_frac; /* 2e-4 */
  float speckle_keep_cost;      /* 0.2 */
  uint32_t fill_holes;          /* false */
  double fill_max_frac;         /* 0.01 */
  float fill_edge_step;         /* 0.06 */
  float fill_max_cost;          /* 1.0 */
} ps_post_params;
void ps_post_params_default(ps_post_params* out);
int ps_postprocess_resident(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_post_params* p,
                            const double* intrinsics, uint64_t* removed, uint64_t* filled);
/* Downloads the current readout planes (after any post-processing) and final costs of `views` at `level` without
 * recomputing the readout. */
int ps_readout_download(ps_session* s, uint32_t level, const uint32_t* views, size_t n, ps_view_state* out);
/* FusionParams of consistency fusion (crates/dense/src/params.rs:264-351) with its handling of leftover pixels
 * (FusionResidual): none; release (the same result as none: fusion.rs:212-214 keeps marks only for adopted points);
 * second pass (fusion.rs:215-218, 540-627): pixels that were neither the reference nor an agreeing pixel of a
 * first-pass point are checked again with the residual tolerances (depth NaN = 0.5 × max_depth_error, normal NaN =
 * 0.67 × max_normal_error_deg) and residual_min_views; a candidate within residual_min_dist_gsd × GSD of a first-pass
 * point is dropped (GSD: the median over views of the median of every 97th valid depth over fx); candidates take
 * their pixels with the smallest candidate number and only those that own their reference pixel are kept. */
#define PS_FUSION_RESIDUAL_NONE 0u
#define PS_FUSION_RESIDUAL_RELEASE 1u
#define PS_FUSION_RESIDUAL_SECOND_PASS 2u
typedef struct ps_fusion_params {
  uint32_t min_consistent_views;   /* 5 */
  uint32_t consistency_num_images; /* 12 (at most 32) */
  uint32_t mark_used;              /* true */
  uint32_t mark_radius;            /* 0 */
  uint32_t inverse_variance;       /* true */
  uint32_t residual;               /* PS_FUSION_RESIDUAL_NONE */
  double sigma_px0;                /* 0.25 */
  double sigma_px_slope;           /* 1.0 */
  double max_reproj_error;         /* 2.0 px */
  double max_depth_error;          /* 0.01 relative */
  double max_normal_error_deg;     /* 10 */
  uint32_t residual_min_views;       /* 2 */
  uint32_t reserved;
  double residual_depth_error;       /* NaN */
  double residual_normal_error_deg;  /* NaN */
  double residual_min_dist_gsd;      /* 0.5 */
  /* free-space visibility filter of the fused cloud (VisibilityParams, crates/dense/src/visibility.rs:50-72,
   * applied as crates/dense/src/densify.rs:544-551 does): a point is projected into up to visibility_check_views
   * candidate views (the overlap lists of its contributing views in order, de-duplicated; at most 64; 0 = off) and
   * removed when at least visibility_min_violations of them see a valid depth beyond it by more than tau (relative)
   * and those outnumber the views that agree within tau. */
  uint32_t visibility_check_views;    /* 0 */
  uint32_t visibility_min_violations; /* 2 */
  double visibility_tau;              /* 0.01 */
  /* bilateral smoothing of the fused points along their normals after the visibility filter (SmoothParams,
   * crates/dense/src/smooth.rs:51-75, applied as densify.rs:552-556 does): smooth_iterations Jacobi passes (0 = off);
   * neighbours within radius = smooth_radius_gsd × GSD whose normal is within smooth_normal_deg move a point along
   * its normal by the weighted mean offset, weights exp(-d²/(2(r/2)²) - dn²/(2σ²)), σ = smooth_sigma_range_gsd × GSD.
   * The exponential is a fixed binary64 sequence (not the platform's), the same in the CPU restatement.  Cells of the
   * radius must stay within ±2^20 of the origin on every axis. */
  uint32_t smooth_iterations;     /* 0 */
  uint32_t reserved2;
  double smooth_radius_gsd;       /* 1.0 */
  double smooth_sigma_range_gsd;  /* 0.25 */
  double smooth_normal_deg;       /* 30 */
} ps_fusion_params;
void ps_fusion_params_default(ps_fusion_params* out);
/* Camera of one view for fusion (DenseView, crates/dense/src/scene.rs): world -> camera x_c = R x_w + t with R
 * row-major, intrinsics k = fx, fy, cx, cy, the representative baseline (median distance to its source centres,
 * crates/dense/src/densify.rs:260-275; 0 = no inverse-variance weight), the point-key image id and the overlap list
 * (views to check, in order; crates/dense/src/densify.rs:519). */
typedef struct ps_fusion_view {
  double k[4];
  double r[9];
  double t[3];
  double baseline;
  uint32_t image_id;
  uint32_t num_overlap;
  const uint32_t* overlap;
} ps_fusion_view;
/* Consistency fusion (crates/dense/src/fusion.rs:219-459) of the readout planes and final costs of `views` at
 * `level`; cams[v] for every session view v (only the listed views are used).  Views are fused in index order.  The
 * point cloud stays in the session; num_points receives its size and num_residual (may be NULL) how many of them
 * the second pass added (FusionOutput::residual).  Colours are the gray image value as u8. */
int ps_fuse_resident(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_fusion_view* cams,
                     const ps_fusion_params* p, uint64_t* num_points, uint64_t* num_residual);
/* Points the visibility filter removed from the last fused cloud (FusionOutput::visibility_removed). */
int ps_fused_visibility_removed(ps_session* s, uint64_t* removed);

/* ScoreFusionOptions (crates/dense/src/fusion_score.rs:56-103).  Score fusion (fuse_scored, fusion_score.rs:314-435):
 * every valid reference pixel is lifted to a point and checked against up to num_neighbors overlap views; a view that
 * agrees in depth and normal contributes c_j·exp(-e²/(2σ_e²))·(1 - exp(-θ²/(2σ_θ²))) (c_j = clamp(1 - cost, 0, 1),
 * e the round-trip reprojection error, θ the angle of the two viewing rays), a view whose surface lies behind the
 * point by more than depth_error costs λ·c_j, and the reference contributes its own c; points scoring at least tau
 * are candidates (weighted means of position, normal, colour).  With mark_used, candidates whose pixels overlap keep
 * only the higher priority (score descending, then view and pixel ascending).  The exponentials and the arc cosine
 * are fixed binary64 sequences shared with the CPU restatement. */
typedef struct ps_score_fusion_params {
  double sigma_e_px;        /* 1.0 */
  double sigma_theta_deg;   /* 2.0 */
  double lambda;            /* 1.0 */
  double tau;               /* 2.0 */
  double depth_error;       /* 0.01 */
  double normal_error_deg;  /* 10 */
  uint32_t num_neighbors;   /* 12 (at most 32) */
  uint32_t mark_used;       /* true */
  uint32_t inverse_variance; /* true */
  uint32_t reserved;
  double sigma_px0;         /* 0.25 */
  double sigma_px_slope;    /* 1.0 */
} ps_score_fusion_params;
void ps_score_fusion_params_default(ps_score_fusion_params* out);
/* Score fusion of the readout planes and final costs of `views` at `level` (cams as for ps_fuse_resident); the
 * cloud replaces the session's fused cloud (ps_fused_points reads it, in the reference's order: view index, then
 * pixel).  `post` (nullable; only its visibility_* and smooth_* fields are read) adds the visibility filter and the
 * smoothing after the fusion, as fuse_depth_maps_with does (crates/dense/src/densify.rs:535-556).  num_points: the
 * adopted points the visibility filter kept. */
int ps_fuse_scored_resident(ps_session* s, uint32_t level, const uint32_t* views, size_t n, const ps_fusion_view* cams,
                            const ps_score_fusion_params* p, const ps_fusion_params* post, uint64_t* num_points);
/* The fused points in the reference's order: after ps_fuse_resident the first pass in ascending point key
 * (image_id << 32) | (row << 16) | col, then the second-pass points in ascending key; after ps_fuse_scored_resident
 * (view index, pixel) order.  Positions and normals 3 floats, colours 3 bytes, keys, the number of contributing views
 * and their indices (ascending; vis_stride >= consistency_num_images + 1, or num_neighbors + 1, entries per point).
 * Any output may be NULL. */
int ps_fused_points(ps_session* s, uint64_t capacity, float* positions, float* normals, uint8_t* colors,
                    uint64_t* keys, uint8_t* vis_counts, uint16_t* vis, uint32_t vis_stride);

/* ---- neighbour views and depth ranges from sparse tracks (crates/dense/src/neighbors.rs:44-186) --------------
 * A view of the sparse model: world -> camera rotation r (row-major) and translation t (DenseView r, t). */
typedef struct ps_sparse_view {
  double r[9];
  double t[3];
} ps_sparse_view;
/* NeighborOptions (crates/dense/src/params.rs:355-369); diversity_decay >= 1 selects plain shared-count order
 * (PairStats::select_all), below 1 the direction-diverse greedy choice (PairStats::select_diverse, as
 * crates/dense/src/densify.rs:224-240 chooses). */
typedef struct ps_neighbor_params {
  uint32_t num_views;                 /* 10: sources kept per view (1..1024) */
  uint32_t direction_bins;            /* 8 */
  double min_triangulation_angle_deg; /* 1.0: pairs whose 75th-percentile angle is below are skipped (0: no test) */
  double diversity_decay;             /* 1.0 */
} ps_neighbor_params;
void ps_neighbor_params_default(ps_neighbor_params* out);
/* PairStats::new + select_all / select_diverse + depth_ranges on the GPU.  Point i has position xyz[3i..3i+3) and
 * the track track_views[track_offsets[i] .. track_offsets[i+1]) (view indices, repeats allowed and counted as the
 * reference counts them).  Outputs: sources[v * num_views + k] for k < num_sources[v] (the rest UINT32_MAX);
 * depth_range[2v], [2v+1] = (0.75·d1%, 1.25·d99%) of the view's positive point depths and has_range[v] = 0 when it
 * has none.  pair_count / pair_angle75 (may be NULL; num_views² entries, index min(a,b)·n + max(a,b)) receive the
 * shared count and the 75th-percentile triangulation angle (radians) of every pair.  At most 4096 views.  Blocking;
 * allocates and frees its own device memory. */
int ps_select_neighbors(int device, const ps_sparse_view* views, uint32_t num_views, const double* xyz,
                        const uint32_t* track_offsets, const uint32_t* track_views, uint64_t num_points,
                        const ps_neighbor_params* p, uint32_t* sources, uint32_t* num_sources, double* depth_range,
                        uint8_t* has_range, uint32_t* pair_count, double* pair_angle75);

/* build_pyramid (crates/dense/src/upsample.rs:46-102) on the GPU: out[0] is the coarsest level, out[levels-1] the
 * input itself; level sizes halve (floor) towards the coarse end; out_k (may be NULL) receives 4 doubles per level
 * (f·0.5, c ← (c + 0.5)·0.5 − 0.5 per step from k).  Blocking; allocates and frees its own device memory. */
int ps_build_pyramid(int device, const uint8_t* gray, uint32_t width, uint32_t height, const double* k,
                     uint32_t levels, uint8_t* const* out, uint32_t* out_w, uint32_t* out_h, double* out_k);

/* DenseOutput::write_ply (crates/dense/src/densify.rs:143-153; crates/core/src/io/ply.rs:82-140, layout
 * XyzNormalRgb): binary little-endian PLY "x y z [nx ny nz] red green blue" (float / uchar), 27 bytes per point with
 * normals.  normals and colors may be NULL (colour 255 then). */
int ps_write_ply(const char* path, uint64_t n, const float* positions, const float* normals, const uint8_t* colors);

/* ---- measurement (no reference counterpart; replaces CUMULUS3D_CUDA_TRACE, crates/cuda/src/patchmatch.rs:780-797) */
typedef enum ps_kernel_kind {
  PS_KERNEL_HALF = 0,
  PS_KERNEL_EVAL = 1,
  PS_KERNEL_FILTER = 2,
  PS_KERNEL_OTHER = 3,
  PS_KERNEL_SWEEP = 4, /* plane sweep of the learned proposal */
  PS_KERNEL_NET = 5,   /* proposal network forward + decode (one event pair per view) */
  PS_KERNEL_KINDS = 6
} ps_kernel_kind;
/* With profiling on, every launch is bracketed by CUDA events on the session stream and half-step / evaluate /
 * filter launches count the NCC window evaluations they perform (each is (2R/step+1)^2 taps). */
int ps_set_profiling(ps_session* s, uint32_t enable);
int ps_kernel_stats(ps_session* s, uint32_t kind, double* total_ms, uint64_t* launches, uint64_t* ncc_windows);
int ps_reset_stats(ps_session* s);
/* With profiling on, the staged half step (PS_TUNE_STAGED) also counts, into stats[8]: [0] NCC windows whose taps
 * read a warp's staged source box, [1] box restages (per warp), and the windows left to the per-lane loops because
 * [2] a footprint was not bounded, [3] the warp's footprint union was too wide or [4] too tall for the box, or [5] too
 * few lanes were active (0 for the other variants and kernel kinds).  Every half-step variant counts into [6] the
 * refinement windows it skipped because the candidate's partial cost had already reached the best cost (the result
 * is the same as evaluating them).  [7] is 0. */
int ps_kernel_staged_stats(ps_session* s, uint32_t kind, uint64_t* stats);
/* Measured FP32 FMA throughput of the device (TFLOP/s, FMA = 2 FLOP) from a register-resident FFMA loop. */
int ps_measure_fp32_peak(int device, double* tflops);
/* Self-check of the numerics contract: compares the kernels' reciprocal with the correctly rounded reciprocal for
 * every binary32 significand at the exponents exp_lo..exp_hi (within -126..127).  *mismatches = the number that
 * differ; first_bad (may be NULL) receives up to 8 differing arguments as bit patterns. */
int ps_check_reciprocal(int device, int exp_lo, int exp_hi, uint64_t* mismatches, uint32_t* first_bad);

#ifdef __cplusplus
}
#endif
#endif /* PATCHSTEREO_H */
