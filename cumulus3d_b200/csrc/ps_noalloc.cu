// ps_median_filter_inplace_noalloc: the 5×5 median plane filter for callers that cannot allocate device memory.
//
// Some callers own their device buffers but may not call cudaMalloc: code running under a host framework whose
// memory pool owns every device allocation, callers working inside a fixed memory budget that forbids growth
// after start-up, or real-time loops where an allocation (and the implicit synchronisation it may bring) is not
// allowed.  The session path (ps_median_filter) copies the input planes into a session-allocated device buffer
// before filtering; this entry point keeps that input copy in a file-scope static device array instead, so the
// call itself allocates nothing.
//
// Limits and sharing rules:
//  * at most PS_NOALLOC_MAX_PIXELS pixels per call (the static array holds that many float4 planes, 32 MiB); every
//    GPU that loads the library reserves this array until the process exits;
//  * every call on a device shares the one array and it keeps the last call's contents; a call first copies its
//    whole input into it and reads only what it copied, so nothing has to start at zero; calls whose work overlaps
//    on the GPU (two streams at once) race on the array;
//  * the first call on a device looks the array's device address up (cudaGetSymbolAddress) with that device
//    current; make that first call before any stream capture.  The address is kept for the life of the process,
//    so it is no longer valid after the caller resets the device (cudaDeviceReset);
//  * `planes` must be device (or managed) memory of `device`: anything else is rejected before any device work;
//  * the call makes `device` current only while it runs and restores the caller's current device before it returns;
//  * it does not run while the calling thread has a CUDA error pending (it returns PS_ECUDA and leaves that error
//    for its owner), so a launch failure it reports is its own.
//
// The arithmetic is the parity build's (this file is compiled with --fmad=false and IEEE division), so the output
// has the same bits as ps_median_filter of a parity-math session on the same planes.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/patchstereo.h"

namespace {

// Input copy of the planes being filtered (nx, ny, nz, d), 2^21 pixels: a 1920×1080 image fits.
static __device__ __align__(256) float4 g_noalloc_scratch[PS_NOALLOC_MAX_PIXELS];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float4* g_scratch_ptr[kMaxDevices] = {};

__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 ray_of(const float* k, int x, int y) {
  return make_float3(((float)x - k[2]) / k[0], ((float)y - k[3]) / k[1], 1.0f);
}

struct Intr {
  float k[4];
};

// 5×5 median plane filter (the rule of crates/dense/src/upsample.rs:192-238 as the GPU kernel states it in
// crates/cuda/src/kernels/patchmatch.cu:805-849): lower median of the depths the valid neighbour planes give on
// this pixel's ray, ties by index; invalid pixels pass through.  Reads `in` (the scratch copy), writes `out`.
// One thread per pixel over a 1-D grid (any image shape within the pixel limit fits the grid's x dimension).
__global__ void __launch_bounds__(256) k_median_noalloc(const float4* __restrict__ in, float4* __restrict__ out, int w,
                                                        int h, Intr K) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)w * h) return;
  const int x = (int)(i % w), y = (int)(i / w);
  const float4 self = in[y * w + x];
  if (!(self.w > 0.f)) {
    out[y * w + x] = self;
    return;
  }
  const float3 rp = ray_of(K.k, x, y);
  float ds[25];
  int qs[25];
  int c = 0;
  for (int qy = max(y - 2, 0); qy < min(y + 3, h); ++qy) {
    for (int qx = max(x - 2, 0); qx < min(x + 3, w); ++qx) {
      const float4 q = in[qy * w + qx];
      if (!(q.w > 0.f)) continue;
      const float3 n = make_float3(q.x, q.y, q.z);
      const float den = dot3(n, rp);
      if (!(den < -1e-6f)) continue;
      const float d = q.w * dot3(n, ray_of(K.k, qx, qy)) / den;
      if (!(d > 0.f) || !isfinite(d)) continue;
      const int qi = qy * w + qx;
      int k = c++;
      while (k > 0 && (ds[k - 1] > d || (ds[k - 1] == d && qs[k - 1] > qi))) {
        ds[k] = ds[k - 1];
        qs[k] = qs[k - 1];
        --k;
      }
      ds[k] = d;
      qs[k] = qi;
    }
  }
  float4 o = self;
  if (c > 0) {
    const int m = (c - 1) / 2;
    const float4 q = in[qs[m]];
    o = make_float4(q.x, q.y, q.z, ds[m]);
  }
  out[y * w + x] = o;
}

}  // namespace

namespace {

// Runs the filter with `device` current (the caller restores its own current device).
int median_noalloc_on(int device, float* planes, uint32_t width, uint32_t height, const float* k, void* stream) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, planes) != cudaSuccess) {
    cudaGetLastError();  // the query's own error
    return PS_EINVAL;
  }
  if (!((a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device)) return PS_EINVAL;
  float4* scratch = nullptr;
  {
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_ptr[device]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
        cudaGetLastError();
        return PS_ECUDA;
      }
      g_scratch_ptr[device] = (float4*)p;
    }
    scratch = g_scratch_ptr[device];
  }
  const cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)width * height;
  if (cudaMemcpyAsync(scratch, planes, n * sizeof(float4), cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
    cudaGetLastError();
    return PS_ECUDA;
  }
  Intr K;
  for (int i = 0; i < 4; ++i) K.k[i] = k[i];
  k_median_noalloc<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(scratch, (float4*)planes, (int)width, (int)height, K);
  if (cudaGetLastError() != cudaSuccess) return PS_ECUDA;
  return PS_OK;
}

}  // namespace

extern "C" int ps_median_filter_inplace_noalloc(int device, float* planes, uint32_t width, uint32_t height,
                                                const float* k, void* stream) {
  if (!planes || !k || width == 0 || height == 0) return PS_EINVAL;
  if (((uintptr_t)planes & 15u) != 0) return PS_EINVAL;  // float4 planes
  if ((uint64_t)width * height > PS_NOALLOC_MAX_PIXELS) return PS_EINVAL;
  if (!(k[0] != 0.0f) || !(k[1] != 0.0f)) return PS_EINVAL;
  if (device < 0 || device >= kMaxDevices) return PS_ENODEV;
  if (cudaPeekAtLastError() != cudaSuccess) return PS_ECUDA;  // the caller's pending error stays pending
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) {
    cudaGetLastError();
    return PS_ENODEV;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return PS_ENODEV;
  }
  const int rc = median_noalloc_on(device, planes, width, height, k, stream);
  if (prev != device && cudaSetDevice(prev) != cudaSuccess) {
    cudaGetLastError();
    return rc == PS_OK ? PS_ECUDA : rc;
  }
  return rc;
}
