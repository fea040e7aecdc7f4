// Internal interface between the proposal network (ps_cnn.cu) and the session runtime (ps_runtime.cu).
#pragma once
#include <cuda_runtime.h>

#include <string>

struct ps_net;

namespace ps_cnn {
// Network forward of `B` inputs of H × W pixels (bf16 NHWC, 48 channels, device) into `out` (f32 NHWC, 8 channels,
// device), enqueued on `st`.  H and W are multiples of 8.  Returns a ps_status; on failure *err holds the message.
int forward_on_stream(ps_net* net, const void* in, int B, int H, int W, float* out, cudaStream_t st, std::string* err);
// Head output -> proposal planes and confidences of an H × W view whose network rows hold Wp pixels; k = fx fy cx cy.
// Adds the number of proposed pixels to *count when count is not null.
cudaError_t launch_decode(const float* o, int Wp, int H, int W, float4* planes, float* conf, float inv_near,
                          float inv_far, float thr, const float* k, unsigned long long* count, cudaStream_t st);
// PS_ETIMEOUT (with a message) when a bounded wait of the tensor-core convolution expired on the current device since
// the counter was last cleared: network outputs computed since then are invalid.  Reads device memory (synchronous).
int conv_health(std::string* err);
// Kernel launches of one inference forward pass (12 convolutions, 3 poolings; upsampling and concatenation are
// fused into the convolutions' input loads).
constexpr int kForwardLaunches = 15;
}  // namespace ps_cnn
